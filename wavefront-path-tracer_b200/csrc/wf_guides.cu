// Denoiser guide buffers: generateFrameGuides (include/renderer/
// device_frame_guides.cuh:6-41, with projectFramePoint from
// include/renderer/frame_guides.cuh:22-44), the per-pixel albedo, normals,
// depth and camera motion that the reference's dataset capture
// (tools/dataset_capture.cu:105-121) exports beside the radiance.
//
// One thread per pixel of the tile: an unjittered primary ray through the
// pixel centre, the closest hit with the material's textured albedo and
// mapped normal, and, given the previous frame's camera, the hit's
// reprojection into that frame and a second closest-hit ray that checks the
// surface was visible there.  The kernel is two closest-hit traversals and a
// 56-byte store per pixel, so it is bound by traversal latency like the
// renderer's trace kernels, and resident warps are what hide it.
#include "wf_renderer.h"
#include "wf_shade.cuh"

#define WF_CUDA(call)                                          \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
    } while (0)

namespace wf {
namespace {

static_assert(sizeof(wf_frame_guide) == 56, "wf_frame_guide is FrameGuide's 14 floats");

// projectFramePoint, include/renderer/frame_guides.cuh:22-44: the pixel
// (integer centres) that `point` projects to; false behind the camera or
// outside the pixel-centre domain (with a 1e-4 margin, then clamped).
WF_DEV bool project_frame_point(const Camera& c, V3 point, uint32_t width, uint32_t height, float& px, float& py) {
    V3 relative = point - c.position;
    float depth = dot(relative, c.forward);
    if (!(depth > 0.0f)) return false;
    float half_height = depth * c.tan_half_fov;
    float u = 0.5f * (dot(relative, c.right) / (half_height * c.aspect_ratio) + 1.0f);
    float v = 0.5f * (1.0f - dot(relative, c.up) / half_height);
    px = u * width - 0.5f;
    py = v * height - 0.5f;
    constexpr float epsilon = 0.0001f;
    float max_x = float(width - 1), max_y = float(height - 1);
    bool inside = px >= -epsilon && py >= -epsilon && px <= max_x + epsilon && py <= max_y + epsilon;
    if (inside) {
        px = fminf(fmaxf(px, 0.0f), max_x);
        py = fminf(fmaxf(py, 0.0f), max_y);
    }
    return inside;
}

// The closest hit of one ray as a SurfaceHit; false on a miss.
WF_DEV bool closest_surface(const DeviceScene& s, V3 o, V3 d, SurfaceHit& sh) {
    TraceState h;
    NoTally tally;
    trace_closest(s, o, d, h, tally);
    return finish_hit(s, o, d, h.t, h.u, h.v, h.prim, h.inst, sh);
}

// Bounded to 8 CTAs of 128 per SM (64 registers, 64 B of spill): a 1080p
// guide frame of the large mesh takes 3.51 ms, against 4.12 ms unbounded (80
// registers, 6 CTAs) and 3.78 ms at 72 registers.
__global__ void __launch_bounds__(128, 8) k_frame_guides(const __grid_constant__ DeviceScene s, Camera camera,
                                                      Camera previous, uint32_t has_previous, uint32_t width,
                                                      uint32_t height, uint32_t x0, uint32_t y0, uint32_t tile_w,
                                                      uint32_t count, wf_frame_guide* out) {
    uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= count) return;
    uint32_t x = x0 + index % tile_w, y = y0 + index / tile_w;
    V3 o, d;
    camera_ray(camera, (x + 0.5f) / width, (y + 0.5f) / height, o, d);
    wf_frame_guide g;
    memset(&g, 0, sizeof(g));
    SurfaceHit sh;
    if (closest_surface(s, o, d, sh)) {
        const Material& m = s.materials[sh.material];
        // getMaterialAlbedo and getMaterialNormal (device_traversal.cuh:363-366,
        // 451-499): the albedo texture (fallback texel 1) through the material's
        // sRGB curve, the normal map when the material has one.
        TexBinding none{};
        none.texture = kInvalid;
        const MaterialTextures* mt = s.material_textures ? &s.material_textures[sh.material] : nullptr;
        float4 texel = sample_binding(s, mt ? mt->slot[kTexAlbedo] : none, sh.uv, sh.uv1,
                                      make_float4(1.0f, 1.0f, 1.0f, 1.0f));
        V3 albedo = hadamard(m.albedo, (m.flags & kMatSpecGlossWorkflow) ? gltf_srgb_to_linear(texel)
                                                                         : srgb_to_linear(texel));
        V3 normal = mt ? material_normal(s, mt->slot[kTexNormal], mt->normal_scale, sh) : sh.normal;
        if (dot(normal, sh.geometric_normal) < 0.0f) normal = -normal;
        g.albedo[0] = albedo.x; g.albedo[1] = albedo.y; g.albedo[2] = albedo.z;
        g.normal[0] = normal.x; g.normal[1] = normal.y; g.normal[2] = normal.z;
        g.geometric_normal[0] = sh.geometric_normal.x;
        g.geometric_normal[1] = sh.geometric_normal.y;
        g.geometric_normal[2] = sh.geometric_normal.z;
        g.depth = dot(sh.position - camera.position, camera.forward);
        g.valid = 1.0f;
        float px, py;
        if (has_previous && project_frame_point(previous, sh.position, width, height, px, py)) {
            g.motion[0] = px - x;
            g.motion[1] = py - y;
            // camera-only motion: the surface counts as seen in the previous
            // frame when the ray through its projection lands on it again
            V3 po, pd;
            camera_ray(previous, (px + 0.5f) / width, (py + 0.5f) / height, po, pd);
            float tolerance = fmaxf(0.001f, length(sh.position - previous.position) * 0.0001f);
            SurfaceHit back;
            if (closest_surface(s, po, pd, back) &&
                length_squared(back.position - sh.position) <= tolerance * tolerance)
                g.history_valid = 1.0f;
        }
    }
    out[index] = g;
}

}  // namespace

static Camera device_camera(const wf_camera& c) {
    Camera d;
    d.position = V3{c.position[0], c.position[1], c.position[2]};
    d.forward = V3{c.forward[0], c.forward[1], c.forward[2]};
    d.right = V3{c.right[0], c.right[1], c.right[2]};
    d.up = V3{c.up[0], c.up[1], c.up[2]};
    d.aspect_ratio = c.aspect_ratio;
    d.tan_half_fov = wfm::tanf(c.vertical_fov * 0.5f);
    return d;
}

wf_status frame_guides(const wf_scene* scene, const wf_camera* camera, const wf_camera* previous, uint32_t width,
                       uint32_t height, uint32_t x, uint32_t y, uint32_t w, uint32_t h, wf_frame_guide* guides,
                       cudaStream_t stream) {
    uint64_t count = uint64_t(w) * h;
    if (count == 0) return WF_OK;
    if (count > 0xffffffffull) return fail(WF_ERR_INVALID_ARG, "tile has more than 2^32 - 1 pixels");
    Camera now = device_camera(*camera);
    Camera before = previous ? device_camera(*previous) : now;
    uint32_t blocks = uint32_t((count + 127) / 128);
    k_frame_guides<<<blocks, 128, 0, stream>>>(scene->view, now, before, previous ? 1u : 0u, width, height, x, y, w,
                                              uint32_t(count), guides);
    WF_CUDA(cudaGetLastError());
    return WF_OK;
}

}  // namespace wf
