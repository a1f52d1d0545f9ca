// Albedo gradients of the production renderer's own image.
//
// wf_diff_* differentiates a reduced integrator of its own.  This file
// replays the renderer's shading itself (shade_path, with the renderer's
// RenderParams) path by path and returns, for a loss whose image adjoint
// the caller supplies, dLoss/d(albedo) of chosen diffuse materials.
//
// Why it is exact per sample.  A diffuse vertex of material a scales the
// path throughput by albedo_a * g (g a scalar: cosine over pdf, the
// continuation's Russian-roulette factor aside) and adds next-event terms
// that are linear in albedo_a; no sampling decision of shade_path reads an
// albedo except Russian roulette's survival probability.  So with the
// random numbers fixed, the derivative of the throughput with respect to
// albedo_m follows the path multiplicatively:
//   dt'_m = dt_m * (t' / t) + [a == m] t' / albedo_a    (componentwise),
// and a term c emitted at a vertex with throughput t has
//   dc_m = c * dt_m / t + [a == m] c / albedo_a.
// The ratios fold in whatever else the vertex multiplied the throughput by
// (glossy and dielectric weights, medium attenuation), which do not depend
// on the parameters.  Russian roulette's 1 / survival is treated as a
// constant ("detached"): the result is then the derivative of the sample's
// estimate for the survival decisions and weights it drew, an unbiased
// estimate of the gradient of the expected image (E[1{u < p} / p] = 1 for
// every p); with Russian roulette off (rr_start_depth >= max_depth) it is
// the exact derivative of the sample's estimate.  The indirect clamp would
// make the terms non-linear in a way the sink cannot see, so it must be 0.
//
// The replay traces with the per-thread traversal and shades with inline
// shadow rays, as the fused persistent kernel does; each pixel adds its
// samples in order, so the image it writes equals wf_render's bit for bit.
#include "wf_renderer.h"
#include "wf_shade.cuh"
#include "wf_wavefront.cuh"

#include <algorithm>
#include <vector>

namespace wf {
namespace {

#define WF_GRAD_CUDA(call)                                        \
    do {                                                          \
        cudaError_t wf_e_ = (call);                               \
        if (wf_e_ != cudaSuccess) return cuda_fail(wf_e_, #call); \
    } while (0)

constexpr uint32_t kGradMaterials = 8;

struct GradParams {
    uint32_t count;
    uint32_t material[kGradMaterials];
};

WF_DEV V3 ratio(V3 a, V3 b) {
    return V3{b.x != 0.0f ? a.x / b.x : 0.0f, b.y != 0.0f ? a.y / b.y : 0.0f, b.z != 0.0f ? a.z / b.z : 0.0f};
}

// InlineSink that also adds each accepted term's contribution to the
// gradient: dLoss/dalbedo_m += adjoint * dc_m.
template <typename Tally>
struct GradSink : InlineSink<Tally> {
    V3 vertex_throughput;  // throughput of the path when the vertex's shading began
    int own;               // parameter index of the vertex's material, or -1
    V3 own_albedo;
    V3 adjoint;            // dLoss/d(pixel radiance)
    const V3* dt;          // dthroughput/dalbedo_m at the vertex
    V3* grad;
    uint32_t count;
    WF_DEV void term(V3 c, int handle) {
        if (!this->may_be_visible(handle)) return;
        this->radiance += c;
        V3 per_throughput = ratio(c, vertex_throughput);
        for (uint32_t m = 0; m < count; ++m) grad[m] += hadamard(adjoint, hadamard(per_throughput, dt[m]));
        if (own >= 0) grad[own] += hadamard(adjoint, ratio(c, own_albedo));
    }
};

// Bounded to 8 CTAs of 128 per SM like the fused persistent kernel, whose
// traversal it shares: four times the resident warps of the unbounded
// build hide more of the dependent node loads than the spills cost.
template <typename Tally, bool kTextures>
__global__ void __launch_bounds__(128, 8) k_albedo_gradient(const __grid_constant__ DeviceScene s,
                                                            const __grid_constant__ RenderParams rp, TileDev tile,
                                                            uint32_t sample_start, uint32_t samples, GradParams gp,
                                                            const float* adjoint, float* image, double* gradient) {
    __shared__ double block_grad[3 * kGradMaterials];
    for (uint32_t k = threadIdx.x; k < 3 * kGradMaterials; k += blockDim.x) block_grad[k] = 0.0;
    __syncthreads();
    V3 grad[kGradMaterials];
    for (uint32_t m = 0; m < kGradMaterials; ++m) grad[m] = V3{0.0f, 0.0f, 0.0f};
    uint32_t pixels = tile.width * tile.height;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < pixels; q += gridDim.x * blockDim.x) {
        uint32_t pixel = (tile.y + q / tile.width) * rp.width + tile.x + q % tile.width;
        V3 adj{adjoint[3 * size_t(pixel)], adjoint[3 * size_t(pixel) + 1], adjoint[3 * size_t(pixel) + 2]};
        float sum_r = 0.0f, sum_g = 0.0f, sum_b = 0.0f;  // the cleared tile, then each sample in order
        for (uint32_t k = 0; k < samples; ++k) {
            Path path;
            init_path(rp, tile, sample_start + k, q, path);
            V3 dt[kGradMaterials];
            for (uint32_t m = 0; m < kGradMaterials; ++m) dt[m] = V3{0.0f, 0.0f, 0.0f};
            GradSink<Tally> sink;
            sink.scene = &s;
            sink.radiance = V3{0.0f, 0.0f, 0.0f};
            sink.requests = 0;
            sink.adjoint = adj;
            sink.dt = dt;
            sink.grad = grad;
            sink.count = gp.count;
            for (uint32_t bounce = 0; bounce < rp.max_depth && bounce < kMaxBounces; ++bounce) {
                TraceState h;
                Tally tally;
                trace_closest(s, path.origin, path.direction, h, tally);
                SurfaceHit sh;
                bool did_hit = finish_hit(s, path.origin, path.direction, h.t, h.u, h.v, h.prim, h.inst, sh);
                sink.own = -1;
                if (did_hit)
                    for (uint32_t m = 0; m < gp.count; ++m)
                        if (gp.material[m] == sh.material) sink.own = int(m);
                if (sink.own >= 0) sink.own_albedo = s.materials[sh.material].albedo;
                V3 before = path.throughput;
                sink.vertex_throughput = before;
                sink.killed = false;
                bool alive = shade_path<GradSink<Tally>, kTextures>(s, rp, path, did_hit, sh, sink);
                if (!alive || sink.killed) break;
                V3 step = ratio(path.throughput, before);
                for (uint32_t m = 0; m < gp.count; ++m) dt[m] = hadamard(dt[m], step);
                if (sink.own >= 0) dt[sink.own] += ratio(path.throughput, sink.own_albedo);
            }
            sum_r += sink.radiance.x;
            sum_g += sink.radiance.y;
            sum_b += sink.radiance.z;
        }
        if (image) {
            image[3 * size_t(pixel)] = sum_r;
            image[3 * size_t(pixel) + 1] = sum_g;
            image[3 * size_t(pixel) + 2] = sum_b;
        }
    }
    for (uint32_t m = 0; m < gp.count; ++m) {
        if (grad[m].x != 0.0f) atomicAdd(&block_grad[3 * m], double(grad[m].x));
        if (grad[m].y != 0.0f) atomicAdd(&block_grad[3 * m + 1], double(grad[m].y));
        if (grad[m].z != 0.0f) atomicAdd(&block_grad[3 * m + 2], double(grad[m].z));
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < 3 * gp.count; k += blockDim.x)
        if (block_grad[k] != 0.0) atomicAdd(&gradient[k], block_grad[k]);
}

template <typename Tally, bool kTextures>
void launch_gradient(uint32_t blocks, cudaStream_t st, const DeviceScene& s, const RenderParams& rp, TileDev tile,
                     uint32_t start, uint32_t count, const GradParams& gp, const float* adjoint, float* image,
                     double* gradient) {
    k_albedo_gradient<Tally, kTextures><<<blocks, 128, 0, st>>>(s, rp, tile, start, count, gp, adjoint, image,
                                                                gradient);
}

}  // namespace
}  // namespace wf

using namespace wf;

// ---------------------------------------------------------------------------
// wf_render_albedo_gradient (include/wavefront.h).  No counterpart in the
// reference, which has no differentiable code.
extern "C" wf_status wf_render_albedo_gradient(wf_renderer* r, uint32_t x, uint32_t y, uint32_t width,
                                               uint32_t height, uint32_t sample_start, uint32_t sample_count,
                                               const uint32_t* materials, uint32_t material_count,
                                               const float* adjoint, float* image, double* gradient) {
    if (!r || !materials || !adjoint || !gradient) return fail(WF_ERR_INVALID_ARG, "null argument");
    const wf_render_config& c = r->config;
    if (width == 0 || height == 0 || x >= c.width || y >= c.height || width > c.width - x || height > c.height - y)
        return fail(WF_ERR_INVALID_ARG, "gradient tile outside the image");
    if (sample_count == 0) return fail(WF_ERR_INVALID_ARG, "empty sample range");
    if (material_count == 0 || material_count > kGradMaterials)
        return fail(WF_ERR_INVALID_ARG, "between 1 and %u parameter materials", kGradMaterials);
    if (r->params.photons.enabled) return fail(WF_ERR_UNSUPPORTED, "albedo gradients need caustics off");
    if (r->params.clamp > 0.0f) return fail(WF_ERR_UNSUPPORTED, "albedo gradients need indirect_clamp = 0");
    if (r->params.debug) return fail(WF_ERR_UNSUPPORTED, "albedo gradients of a debug view");
    const DeviceScene& s = r->scene->view;
    std::vector<Material> host(s.material_count);
    WF_GRAD_CUDA(cudaMemcpyAsync(host.data(), s.materials, sizeof(Material) * host.size(), cudaMemcpyDeviceToHost,
                                 r->stream));
    WF_GRAD_CUDA(cudaStreamSynchronize(r->stream));
    GradParams gp{};
    gp.count = material_count;
    for (uint32_t m = 0; m < material_count; ++m) {
        uint32_t k = materials[m];
        if (k >= host.size()) return fail(WF_ERR_INVALID_ARG, "parameter material %u out of range", k);
        const Material& mat = host[k];
        if (mat.type != kDiffuse || mat.metallic > 0.5f || (mat.flags & (kMatGltfPbr | kMatTextured)))
            return fail(WF_ERR_UNSUPPORTED, "parameter material %u is not an untextured diffuse material", k);
        if (!(mat.albedo.x > 0.0f && mat.albedo.y > 0.0f && mat.albedo.z > 0.0f))
            return fail(WF_ERR_UNSUPPORTED, "parameter material %u has a zero albedo channel", k);
        for (uint32_t j = 0; j < m; ++j)
            if (materials[j] == k) return fail(WF_ERR_INVALID_ARG, "parameter material %u listed twice", k);
        gp.material[m] = k;
    }
    cudaStream_t st = r->stream;
    TileDev tile{x, y, width, height, 0};
    uint32_t pixels = width * height;
    uint32_t blocks = (pixels + 127) / 128;  // one pixel per thread; the hardware balances the CTAs
    // The variants of the fused persistent kernel: the alpha test only when
    // some material is alpha-textured, the texture code only when one is
    // textured.
    if (!r->opaque)
        launch_gradient<NoTally, true>(blocks, st, s, r->params, tile, sample_start, sample_count, gp, adjoint, image,
                                       gradient);
    else if (r->textured)
        launch_gradient<Opaque<NoTally>, true>(blocks, st, s, r->params, tile, sample_start, sample_count, gp,
                                               adjoint, image, gradient);
    else
        launch_gradient<Opaque<NoTally>, false>(blocks, st, s, r->params, tile, sample_start, sample_count, gp,
                                                adjoint, image, gradient);
    WF_GRAD_CUDA(cudaGetLastError());
    WF_GRAD_CUDA(cudaStreamSynchronize(st));
    return WF_OK;
}
