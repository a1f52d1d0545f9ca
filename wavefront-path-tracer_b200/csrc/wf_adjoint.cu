// Differentiable rendering by path replay (no counterpart in the reference).
//
// Model.  Every non-emissive triangle t has its own Oren-Nayar BRDF
// (Oren and Nayar, "Generalization of Lambert's reflectance model",
// SIGGRAPH 1994; the qualitative model
//   f = albedo/pi * (A + B * max(0, cos(phi_i - phi_o)) * sin(alpha) * tan(beta)),
//   A = 1 - 0.5 s^2 / (s^2 + 0.33),  B = 0.45 s^2 / (s^2 + 0.09),
// with s the roughness in radians); emissive triangles emit their material
// emission times one global scale.  Direct light comes from next-event
// estimation over the scene's triangle lights only (a continuation ray that
// reaches a light adds nothing), continuations are cosine-sampled, and there
// is no Russian roulette and no clamp.  The parameter index of a triangle is
// its index in its mesh (or triangle list) as given to wf_scene_create.
//
// Gradients.  No sampling decision depends on the parameters, so the
// derivative of each path's estimate with the path held fixed is exact for
// that path, and its expectation is the derivative of the image.  A path's
// radiance is a sum of terms T_j; each continuation weight w_m and each
// next-event term multiplies in one BRDF value.  With U the path's total
// radiance and P_m the sum of terms up to vertex m, the terms after vertex m
// sum to U - P_m, so
//   dU/dtheta(t_m) += (U - P_m) * (dw_m/dtheta) / w_m + T_m * (df_m/dtheta) / f_m.
// The adjoint kernel replays each path twice from its RNG key (pass A: U;
// pass B: the sum above), instead of storing paths: memory is O(pixels).
// Gradients are accumulated with double atomics.
#include "wf_wavefront.cuh"

#include <algorithm>
#include <cstring>

namespace wf {

struct DiffSettings {
    Camera camera;
    uint32_t width, height;  // full image (camera and RNG pixel index)
    uint32_t x, y, w, h;     // rendered crop
    uint32_t spp, sample_start, max_depth, rng;
    uint32_t parameters;     // triangles with parameters
};

struct DiffParams {
    const float* albedo;     // 3 per parameter index
    const float* roughness;  // 1 per parameter index (radians)
    float emission_scale;
};

struct DiffGrads {
    double* albedo;
    double* roughness;
    double* emission_scale;
};

namespace {

// Oren-Nayar shape factor and its derivative with respect to the roughness.
struct OrenNayar {
    float value;   // A + B * g
    float d_sigma; // dA/ds + dB/ds * g
};

WF_DEV OrenNayar oren_nayar(V3 n, V3 wo, V3 wi, float sigma) {
    float cos_i = fminf(1.0f, fmaxf(0.0f, dot(n, wi)));
    float cos_o = fminf(1.0f, fmaxf(0.0f, dot(n, wo)));
    float sin_i = sqrtf(fmaxf(0.0f, 1.0f - cos_i * cos_i));
    float sin_o = sqrtf(fmaxf(0.0f, 1.0f - cos_o * cos_o));
    float g = 0.0f;
    if (sin_i > 1e-4f && sin_o > 1e-4f) {
        V3 ti = (wi - n * cos_i) / sin_i;
        V3 to = (wo - n * cos_o) / sin_o;
        float cos_phi = fmaxf(0.0f, dot(ti, to));
        // alpha = max(theta_i, theta_o), beta = min(theta_i, theta_o)
        float sin_alpha = cos_i < cos_o ? sin_i : sin_o;
        float tan_beta = cos_i < cos_o ? sin_o / fmaxf(cos_o, 1e-4f) : sin_i / fmaxf(cos_i, 1e-4f);
        g = cos_phi * sin_alpha * tan_beta;
    }
    float s2 = sigma * sigma;
    float a = 1.0f - 0.5f * s2 / (s2 + 0.33f);
    float b = 0.45f * s2 / (s2 + 0.09f);
    float da = -0.33f * sigma / ((s2 + 0.33f) * (s2 + 0.33f));
    float db = 0.081f * sigma / ((s2 + 0.09f) * (s2 + 0.09f));
    return OrenNayar{a + b * g, da + db * g};
}

constexpr float kInvPi = 0.318309886183790671538f;

// Cosine-weighted direction about n from two uniform numbers (Malley's
// method: a uniform point on the disk lifted to the hemisphere).
WF_DEV V3 sample_cosine_hemisphere_uv(V3 n, float u1, float u2) {
    constexpr float two_pi = 6.28318530718f;
    float radius = sqrtf(u1);
    float phi = two_pi * u2;
    float x = radius * wfm::cosf(phi);
    float y = radius * wfm::sinf(phi);
    float z = sqrtf(1.0f - u1);
    V3 helper = fabsf(n.x) > 0.1f ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
    V3 tangent = normalize(cross(helper, n));
    V3 bitangent = cross(n, tangent);
    return normalize(tangent * x + bitangent * y + n * z);
}

WF_DEV uint32_t parameter_index(const DeviceScene& s, uint32_t prim) {
    TriVerts tri = load_triangle(s, hit_index(prim));
    return tri.index_flags & kTriIndexMask;
}

// Gradient contributions of one vertex, summed over the lanes of a warp
// that hit the same triangle (all 32 lanes call this together).  One lane
// per triangle adds the sums with double atomics.
WF_DEV void flush_vertex(uint32_t key, float4 value, float4* warp_buffer, const DiffGrads& G) {
    uint32_t lane = threadIdx.x & 31;
    unsigned peers = __match_any_sync(0xffffffffu, key);
    warp_buffer[lane] = value;
    __syncwarp();
    if (key != kInvalid && lane == uint32_t(__ffs(peers) - 1)) {
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (unsigned m = peers; m; m &= m - 1) {
            float4 v = warp_buffer[__ffs(m) - 1];
            sum.x += v.x;
            sum.y += v.y;
            sum.z += v.z;
            sum.w += v.w;
        }
        if (sum.x != 0.0f) atomicAdd(&G.albedo[3 * key], double(sum.x));
        if (sum.y != 0.0f) atomicAdd(&G.albedo[3 * key + 1], double(sum.y));
        if (sum.z != 0.0f) atomicAdd(&G.albedo[3 * key + 2], double(sum.z));
        if (sum.w != 0.0f) atomicAdd(&G.roughness[key], double(sum.w));
    }
    __syncwarp();
}

// One path of pixel (px, py), sample `sample`.  kAdjoint = false: returns
// the path radiance at emission scale 1 (the image multiplies by the scale).
// kAdjoint = true: `total` is that radiance from the first replay; adds
// delta * dU/dtheta to the gradients and returns the replayed radiance.  In
// adjoint mode all 32 lanes of the warp call it together (`alive` false for
// lanes without a path) and run the same number of vertex steps.
// Tally: the traversal variant (Opaque<NoTally> when no material of the scene
// is alpha-textured, which drops the per-candidate alpha test).
template <bool kAdjoint, typename Tally>
WF_DEV V3 diff_path(const DeviceScene& s, const DiffParams& P, const DiffSettings& cfg, uint32_t px, uint32_t py,
                    uint32_t sample, bool alive, V3 total, V3 delta, const DiffGrads& G, float4* warp_buffer,
                    uint32_t* error) {
    V3 o{0.0f, 0.0f, 0.0f}, d{0.0f, 0.0f, 1.0f};
    uint64_t rng = 0;
    if (alive) {
        uint32_t pixel = py * cfg.width + px;
        rng = make_rng_state(pixel_rng_key(pixel, sample, cfg.rng), cfg.rng);
        float u = (float(px) + random_float(rng, cfg.rng)) / float(cfg.width);
        float v = (float(py) + random_float(rng, cfg.rng)) / float(cfg.height);
        camera_ray(cfg.camera, u, v, o, d);
    }
    V3 beta{1.0f, 1.0f, 1.0f};
    V3 sum{0.0f, 0.0f, 0.0f};  // terms so far, at emission scale 1
    Tally tally;
    for (uint32_t depth = 0; depth < cfg.max_depth; ++depth) {
        if (!kAdjoint && !alive) break;
        uint32_t key = kInvalid;
        float4 contribution = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        do {
            if (!alive) break;
            alive = false;  // set again below when the path continues
            TraceState h;
            trace_closest(s, o, d, h, tally);
            SurfaceHit sh;
            if (!finish_hit(s, o, d, h.t, h.u, h.v, h.prim, h.inst, sh)) break;
            const Material& m = s.materials[sh.material];
            if (m.type == kEmissive) {
                if (depth == 0) sum += hadamard(beta, m.emission);
                break;
            }
            if (hit_kind(h.prim) == kHitSphere) break;  // spheres carry no parameters: they absorb
            uint32_t k = parameter_index(s, h.prim);
            if (k >= cfg.parameters) {
                atomicOr(error, 1u);
                break;
            }
            V3 albedo{P.albedo[3 * k], P.albedo[3 * k + 1], P.albedo[3 * k + 2]};
            float sigma = P.roughness[k];
            V3 gn = sh.geometric_normal;
            V3 n = sh.normal;
            if (dot(n, gn) < 0.0f) n = -n;
            V3 wo = -d;
            // next event: one triangle light picked by the alias table, one point on it
            V3 nee_albedo_free{0.0f, 0.0f, 0.0f};  // term without the albedo factor
            float nee_dsigma = 0.0f;               // d(term)/d(sigma) / term
            if (s.light_count > 0) {
                uint32_t candidate = min(uint32_t(random_float(rng, cfg.rng) * s.light_count), s.light_count - 1);
                const Light* cl = &s.lights[candidate];
                uint32_t li = random_float(rng, cfg.rng) < cl->alias_probability ? candidate : cl->alias;
                const Light& light = s.lights[li];
                float root_u = sqrtf(random_float(rng, cfg.rng));
                float lv = random_float(rng, cfg.rng);
                V3 lp = (1.0f - root_u) * light.v0 + root_u * (1.0f - lv) * light.v1 + root_u * lv * light.v2;
                V3 to_light = lp - sh.position;
                float dist2 = length_squared(to_light);
                float dist = sqrtf(dist2);
                V3 wl = to_light / dist;
                float cos_g = dot(gn, wl), cos_s = dot(n, wl), cos_l = dot(light.normal, -wl);
                if (cos_g > 0.0f && cos_s > 0.0f && cos_l > 0.0f) {
                    V3 so = offset_ray_origin(sh.position, gn, wl, sh.t);
                    V3 st = offset_ray_origin(lp, light.normal, -wl, dist);
                    V3 seg = st - so;
                    float sd = length(seg);
                    if (sd > kRayMinDistance && !trace_any(s, so, seg / sd, sd - kRayMinDistance, tally)) {
                        OrenNayar on = oren_nayar(n, wo, wl, sigma);
                        float geometry = cos_l * light.area / (dist2 * light.selection_pdf);
                        const Material& lm = s.materials[light.material];
                        nee_albedo_free = hadamard(beta, lm.emission) * (on.value * kInvPi * cos_s * geometry);
                        nee_dsigma = on.value > 0.0f ? on.d_sigma / on.value : 0.0f;
                        sum += hadamard(albedo, nee_albedo_free);
                    }
                }
            }
            // continuation: cosine-weighted about the shading normal
            float r1 = random_float(rng, cfg.rng), r2 = random_float(rng, cfg.rng);
            V3 wi = sample_cosine_hemisphere_uv(n, r1, r2);
            bool continues = depth + 1 < cfg.max_depth && dot(wi, gn) > 0.0f;
            OrenNayar on = continues ? oren_nayar(n, wo, wi, sigma) : OrenNayar{0.0f, 0.0f};
            if constexpr (kAdjoint) {
                // terms after this vertex all carry this vertex's continuation weight
                V3 after = total - sum;
                V3 ga{0.0f, 0.0f, 0.0f};
                float gs = 0.0f;
                if (continues) {
                    ga = V3{albedo.x > 0.0f ? after.x / albedo.x : 0.0f, albedo.y > 0.0f ? after.y / albedo.y : 0.0f,
                            albedo.z > 0.0f ? after.z / albedo.z : 0.0f};
                    gs = on.value > 0.0f ? dot(delta, after) * (on.d_sigma / on.value) : 0.0f;
                }
                ga += nee_albedo_free;
                gs += dot(delta, hadamard(albedo, nee_albedo_free)) * nee_dsigma;
                V3 dga = hadamard(delta, ga);
                key = k;
                contribution = make_float4(dga.x, dga.y, dga.z, gs);
            }
            if (!continues) break;
            beta = hadamard(beta, albedo * on.value);
            o = offset_ray_origin(sh.position, gn, wi, sh.t);
            d = wi;
            alive = true;
        } while (false);
        if constexpr (kAdjoint) flush_vertex(key, contribution, warp_buffer, G);
    }
    return sum;
}

// Both kernels trace one path per thread; bounded to 8 CTAs of 128 per SM
// (64 registers) they keep enough warps resident to hide traversal latency.
// Inverse-rendering config (512x512, 32 spp), with the opaque traversal:
// forward 58.9 -> 42.0 ms, adjoint 182 -> 124.5 ms against the unbounded
// kernels (138 and 168 registers, 3 CTAs per SM).
template <typename Tally>
__global__ void __launch_bounds__(128, 8) k_diff_forward(const __grid_constant__ DeviceScene s, DiffParams P,
                                                         DiffSettings cfg, float* image, uint32_t* error) {
    uint32_t n = cfg.w * cfg.h;
    DiffGrads none{};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t px = cfg.x + i % cfg.w, py = cfg.y + i / cfg.w;
        V3 acc{0.0f, 0.0f, 0.0f};
        for (uint32_t k = 0; k < cfg.spp; ++k)
            acc += diff_path<false, Tally>(s, P, cfg, px, py, cfg.sample_start + k, true, V3{}, V3{}, none, nullptr,
                                           error);
        float scale = P.emission_scale / float(cfg.spp);
        float* out = image + 3 * (size_t(py) * cfg.width + px);
        out[0] = acc.x * scale;
        out[1] = acc.y * scale;
        out[2] = acc.z * scale;
    }
}

// d_image: dLoss/dImage (image = mean over samples of emission_scale * U).
// Each warp takes up to 32 samples of one pixel, so the lanes of a warp
// mostly hit the same triangles and their gradients merge before the
// atomics (flush_vertex).
template <typename Tally>
__global__ void __launch_bounds__(128, 8) k_diff_backward(const __grid_constant__ DeviceScene s, DiffParams P,
                                                          DiffSettings cfg, const float* d_image, DiffGrads G,
                                                          uint32_t* error) {
    __shared__ float4 buffers[4][32];
    float4* warp_buffer = buffers[threadIdx.x >> 5];
    uint32_t lane = threadIdx.x & 31;
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t chunks = (cfg.spp + 31) / 32;
    uint32_t items = cfg.w * cfg.h * chunks;
    double d_scale = 0.0;
    DiffGrads none{};
    for (uint32_t item = warp; item < items; item += warps) {
        uint32_t i = item / chunks, chunk = item % chunks;
        uint32_t px = cfg.x + i % cfg.w, py = cfg.y + i / cfg.w;
        const float* g = d_image + 3 * (size_t(py) * cfg.width + px);
        V3 grad_pixel{g[0], g[1], g[2]};
        if (grad_pixel.x == 0.0f && grad_pixel.y == 0.0f && grad_pixel.z == 0.0f) continue;  // uniform per warp
        uint32_t k = chunk * 32 + lane;
        bool alive = k < cfg.spp;
        uint32_t sample = cfg.sample_start + k;
        // the image is scale/spp * sum U: dLoss/dU = dLoss/dImage * scale / spp
        V3 delta = grad_pixel * (P.emission_scale / float(cfg.spp));
        V3 total{0.0f, 0.0f, 0.0f};
        if (alive) total = diff_path<false, Tally>(s, P, cfg, px, py, sample, true, V3{}, V3{}, none, nullptr, error);
        diff_path<true, Tally>(s, P, cfg, px, py, sample, alive, total, delta, G, warp_buffer, error);
        if (alive) d_scale += double(dot(grad_pixel, total)) / double(cfg.spp);
    }
    for (int off = 16; off > 0; off >>= 1) d_scale += __shfl_down_sync(0xffffffffu, d_scale, off);
    if (lane == 0 && d_scale != 0.0) atomicAdd(G.emission_scale, d_scale);
}

// Error flag of the differentiable kernels (a parameter index out of range).
static __device__ uint32_t g_diff_error;

wf_status diff_setup(const wf_scene* scene, const wf_camera* camera, const wf_diff_config* c, DiffSettings& cfg,
                     uint32_t** error) {
    if (!scene || !camera || !c) return fail(WF_ERR_INVALID_ARG, "null argument");
    if (c->width == 0 || c->height == 0 || c->spp == 0 || c->max_depth == 0 || c->max_depth > kMaxBounces)
        return fail(WF_ERR_INVALID_ARG, "empty image, no samples or depth outside [1, %d]", kMaxBounces);
    if (c->rng > WF_RNG_PCG32) return fail(WF_ERR_INVALID_ARG, "unknown rng strategy");
    if (c->parameter_count == 0) return fail(WF_ERR_INVALID_ARG, "no parameters");
    uint32_t cw = c->crop_width ? c->crop_width : c->width, ch = c->crop_height ? c->crop_height : c->height;
    if (c->crop_x >= c->width || c->crop_y >= c->height || cw > c->width - c->crop_x || ch > c->height - c->crop_y)
        return fail(WF_ERR_INVALID_ARG, "crop outside the image");
    cfg = DiffSettings{};
    cfg.camera.position = V3{camera->position[0], camera->position[1], camera->position[2]};
    cfg.camera.forward = V3{camera->forward[0], camera->forward[1], camera->forward[2]};
    cfg.camera.right = V3{camera->right[0], camera->right[1], camera->right[2]};
    cfg.camera.up = V3{camera->up[0], camera->up[1], camera->up[2]};
    cfg.camera.aspect_ratio = camera->aspect_ratio;
    cfg.camera.tan_half_fov = wfm::tanf(camera->vertical_fov * 0.5f);
    cfg.width = c->width;
    cfg.height = c->height;
    cfg.x = c->crop_x;
    cfg.y = c->crop_y;
    cfg.w = cw;
    cfg.h = ch;
    cfg.spp = c->spp;
    cfg.sample_start = c->sample_start;
    cfg.max_depth = c->max_depth;
    cfg.rng = c->rng;
    cfg.parameters = c->parameter_count;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_diff_error);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(diff error flag)");
    *error = static_cast<uint32_t*>(p);
    return WF_OK;
}

wf_status diff_finish(uint32_t* error, cudaStream_t st) {
    uint32_t flag = 0;
    cudaError_t e = cudaMemcpyAsync(&flag, error, sizeof(flag), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "differentiable render");
    if (flag) return fail(WF_ERR_INVALID_ARG, "a hit triangle's parameter index is not below parameter_count");
    return WF_OK;
}

uint32_t diff_grid(uint32_t n) { return std::max(1u, std::min((n + 127) / 128, 148u * 16u)); }

}  // namespace
}  // namespace wf

using namespace wf;

extern "C" wf_status wf_diff_forward(const wf_scene* scene, const wf_camera* camera, const wf_diff_config* config,
                                     const float* albedo, const float* roughness, float emission_scale, float* image,
                                     void* stream) {
    DiffSettings cfg;
    uint32_t* error = nullptr;
    if (wf_status e = diff_setup(scene, camera, config, cfg, &error)) return e;
    if (!albedo || !roughness || !image) return fail(WF_ERR_INVALID_ARG, "null device pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t ce = cudaMemsetAsync(error, 0, sizeof(uint32_t), st);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemsetAsync");
    DiffParams P{albedo, roughness, emission_scale};
    if (scene->alpha_textures)
        k_diff_forward<NoTally><<<diff_grid(cfg.w * cfg.h), 128, 0, st>>>(scene->view, P, cfg, image, error);
    else
        k_diff_forward<Opaque<NoTally>><<<diff_grid(cfg.w * cfg.h), 128, 0, st>>>(scene->view, P, cfg, image, error);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return cuda_fail(ce, "k_diff_forward");
    return diff_finish(error, st);
}

extern "C" wf_status wf_diff_backward(const wf_scene* scene, const wf_camera* camera, const wf_diff_config* config,
                                      const float* albedo, const float* roughness, float emission_scale,
                                      const float* d_image, double* d_albedo, double* d_roughness,
                                      double* d_emission_scale, void* stream) {
    DiffSettings cfg;
    uint32_t* error = nullptr;
    if (wf_status e = diff_setup(scene, camera, config, cfg, &error)) return e;
    if (!albedo || !roughness || !d_image || !d_albedo || !d_roughness || !d_emission_scale)
        return fail(WF_ERR_INVALID_ARG, "null device pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t ce = cudaMemsetAsync(error, 0, sizeof(uint32_t), st);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemsetAsync");
    DiffParams P{albedo, roughness, emission_scale};
    DiffGrads G{d_albedo, d_roughness, d_emission_scale};
    uint32_t items = cfg.w * cfg.h * ((cfg.spp + 31) / 32);  // one warp each
    uint32_t blocks = std::max(1u, std::min((items + 3) / 4, 148u * 16u));
    if (scene->alpha_textures)
        k_diff_backward<NoTally><<<blocks, 128, 0, st>>>(scene->view, P, cfg, d_image, G, error);
    else
        k_diff_backward<Opaque<NoTally>><<<blocks, 128, 0, st>>>(scene->view, P, cfg, d_image, G, error);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return cuda_fail(ce, "k_diff_backward");
    return diff_finish(error, st);
}
