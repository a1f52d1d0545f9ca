// C ABI entry points (include/wavefront.h).
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <vector>
#include <fstream>
#include <memory>

#include "wf_renderer.h"
#include "wf_bvh_gpu.h"

namespace wf {
const char* last_error_text();

namespace {
// wf_test_fail_allocation: allocations left before the injected failure
// (-1 = none armed).
std::atomic<long long> g_fail_allocation{-1};
}  // namespace

cudaError_t device_alloc(void** p, size_t bytes) {
    long long left = g_fail_allocation.load();
    while (left >= 0) {
        if (g_fail_allocation.compare_exchange_weak(left, left - 1)) {
            if (left == 0) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
}
}  // namespace wf

extern "C" void wf_test_fail_allocation(int64_t after) { wf::g_fail_allocation.store(after < 0 ? -1 : after); }

using namespace wf;

#define WF_CUDA(call)                                              \
    do {                                                           \
        cudaError_t wf_e_ = (call);                                \
        if (wf_e_ != cudaSuccess) return cuda_fail(wf_e_, #call); \
    } while (0)

namespace {

template <typename T>
cudaError_t upload(wf_scene* s, std::vector<void*>& list, uint64_t& bytes, const T** out, const std::vector<T>& v) {
    *out = nullptr;
    if (v.empty()) return cudaSuccess;
    void* p = nullptr;
    size_t n = sizeof(T) * v.size();
    cudaError_t e = device_alloc(&p, n);
    if (e != cudaSuccess) return e;
    list.push_back(p);
    bytes += n;
    e = cudaMemcpy(p, v.data(), n, cudaMemcpyHostToDevice);
    *out = static_cast<const T*>(p);
    (void)s;
    return e;
}

void free_list(std::vector<void*>& list) {
    for (void* p : list) cudaFree(p);
    list.clear();
}

// Checkpoint header, src/renderer/render_checkpoint.cpp:17-27 (v3).
struct CheckpointHeader {
    char magic[8];
    uint32_t version;
    uint32_t width;
    uint32_t height;
    uint32_t sample_index;
    uint64_t fingerprint;
};
static_assert(sizeof(CheckpointHeader) == 32, "checkpoint header layout");
constexpr char kMagic[8] = {'P', 'T', 'C', 'H', 'K', 'P', 'T', '1'};
constexpr uint32_t kCheckpointVersion = 3;

wf_status write_checkpoint(const char* path, const float* rgb, uint32_t width, uint32_t height, uint32_t sample,
                           uint64_t fingerprint) {
    CheckpointHeader header{};
    std::memcpy(header.magic, kMagic, 8);
    header.version = kCheckpointVersion;
    header.width = width;
    header.height = height;
    header.sample_index = sample;
    header.fingerprint = fingerprint;
    std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream out(tmp, std::ios::binary | std::ios::trunc);
        if (!out) return fail(WF_ERR_IO, "Could not open checkpoint for writing: %s", tmp.c_str());
        out.write(reinterpret_cast<const char*>(&header), sizeof(header));
        out.write(reinterpret_cast<const char*>(rgb), std::streamsize(sizeof(float) * 3 * size_t(width) * height));
        out.close();
        if (!out) return fail(WF_ERR_IO, "Could not write checkpoint: %s", tmp.c_str());
    }
    if (std::rename(tmp.c_str(), path) != 0) return fail(WF_ERR_IO, "Could not replace checkpoint: %s", path);
    return WF_OK;
}

}  // namespace

extern "C" {

const char* wf_last_error(void) { return last_error_text(); }
const char* wf_version(void) { return "wavefront-b200 1.0"; }

void wf_material_default(wf_material* m, uint32_t type) {
    std::memset(m, 0, sizeof(*m));
    m->type = type;
    m->ior = 1.0f;
    m->attenuation_color[0] = m->attenuation_color[1] = m->attenuation_color[2] = 1.0f;
    m->volume_density = 1.0f;
    m->opacity = 1.0f;
    m->alpha_cutoff = 0.5f;
    m->specular[0] = m->specular[1] = m->specular[2] = 1.0f;
    m->glossiness = 1.0f;
    m->specular_weight = 1.0f;
    m->specular_color[0] = m->specular_color[1] = m->specular_color[2] = 1.0f;
}

void wf_render_config_default(wf_render_config* c, uint32_t width, uint32_t height) {
    std::memset(c, 0, sizeof(*c));
    c->width = width;
    c->height = height;
    c->max_depth = 32;
    c->rr_start_depth = 12;
    c->mode = WF_MODE_GRAPH;
    c->rng = WF_RNG_XORSHIFT32;
    c->indirect_clamp = 10.0f;
    c->caustic_gather = 1;
    c->photon_count = 1048576;
    c->photon_max_depth = 8;
    c->gather_radius = 0.06f;
    c->photon_grid_min[0] = -2.5f; c->photon_grid_min[1] = -1.0f; c->photon_grid_min[2] = -2.5f;
    c->photon_grid_max[0] = 2.5f;  c->photon_grid_max[1] = 3.0f;  c->photon_grid_max[2] = 2.5f;
    c->photon_grid_resolution = 64;
    c->photon_seed = 0x13579bdfu;
    c->profile_queues = 1;
}

wf_status wf_scene_create(const wf_scene_desc* desc, wf_scene** out) {
    if (!out) return fail(WF_ERR_INVALID_ARG, "null output");
    *out = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    HostScene h;
    if (wf_status e = build_host_scene(desc, h)) return e;
    auto s = std::make_unique<wf_scene>();
    WF_CUDA(cudaGetDevice(&s->device));
    DeviceScene& v = s->view;
    auto& L = s->allocations;
    uint64_t& B = s->device_bytes;
    cudaError_t e = cudaSuccess;
    auto up = [&](auto** dst, const auto& vec) {
        if (e == cudaSuccess) e = upload(s.get(), L, B, dst, vec);
    };
    up(&v.triangles, h.triangles);
    up(&v.normals, h.normals);
    up(&v.nodes, h.nodes);
    up(&v.blases, h.blases);
    up(&v.instances, h.instances);
    up(&v.mesh_linear, h.mesh_linear);
    up(&v.tlas_leaves, h.tlas_leaves);
    up(&v.spheres, h.spheres);
    up(&v.sphere_materials, h.sphere_materials);
    up(&v.direct_spheres, h.direct_spheres);
    up(&v.direct_instances, h.direct_instances);
    up(&v.materials, h.materials);
    up(&v.material_textures, h.material_textures);
    up(&v.texels, h.texels);
    up(&v.textures, h.textures);
    up(&v.tri_attr, h.tri_attr);
    up(&v.lights, h.lights);
    up(&v.punctual, h.punctual);
    if (e != cudaSuccess) {
        free_list(L);
        return e == cudaErrorMemoryAllocation ? fail(WF_ERR_OOM, "scene upload: out of device memory")
                                              : cuda_fail(e, "scene upload");
    }
    v.env = Environment{};
    v.tlas = h.tlas;
    v.direct_bvh = h.direct_bvh;
    v.static_first = h.static_first;
    v.static_count = h.static_count;
    v.direct_first = h.direct_first;
    v.direct_count = h.direct_count;
    v.direct_sphere_count = uint32_t(h.direct_spheres.size());
    v.direct_instance_count = uint32_t(h.direct_instances.size());
    v.instance_count = uint32_t(h.instances.size());
    v.material_count = uint32_t(h.materials.size());
    for (const Material& m : h.materials) s->material_categories |= 1u << material_category(m);
    v.light_count = uint32_t(h.lights.size());
    v.punctual_count = uint32_t(h.punctual.size());
    v.directional_count = h.directional_count;
    v.any_alpha_reject = h.any_alpha_reject ? 1u : 0u;
    v.texture_count = uint32_t(h.textures.size());
    v.use_normal_maps = h.use_normal_maps ? 1u : 0u;
    v.normal_map_min_cosine = h.normal_map_min_cosine;
    v.black_background = h.black_background ? 1u : 0u;
    v.ignore_direct_light_occlusion = h.ignore_occlusion ? 1u : 0u;
    s->light_count = v.light_count;
    s->tlas_leaf_count = uint32_t(h.tlas_leaves.size());
    s->blas_count = uint32_t(h.blases.size());
    s->material_count = v.material_count;
    s->bounds = h.bounds;
    s->gpu_bvh_builds = h.gpu_bvh_builds;
    s->alpha_textures = h.alpha_textures;
    s->textured = h.textured;
    s->bvh_build_ms = h.bvh_build_ms;
    s->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = s.release();
    return WF_OK;
}

// No counterpart in the reference, whose materials are fixed at upload.
// Overwrites the albedo of each listed material in the device scene, in
// place: renderers made from the scene read it at their next render
// (captured graphs keep the materials' address, not their contents).
wf_status wf_scene_set_albedos(wf_scene* s, const uint32_t* materials, const float* rgb, uint32_t count) {
    if (!s || (count && (!materials || !rgb))) return fail(WF_ERR_INVALID_ARG, "null argument");
    for (uint32_t k = 0; k < count; ++k) {
        if (materials[k] >= s->material_count)
            return fail(WF_ERR_INVALID_ARG, "material %u out of range (%u materials)", materials[k], s->material_count);
        for (int c = 0; c < 3; ++c)
            if (!std::isfinite(rgb[3 * k + c])) return fail(WF_ERR_INVALID_ARG, "albedo of material %u is not finite",
                                                            materials[k]);
    }
    WF_CUDA(cudaDeviceSynchronize());  // no kernel may be reading the materials
    for (uint32_t k = 0; k < count; ++k) {
        // the scene owns the array; the view only exposes it read-only to kernels
        char* dst = const_cast<char*>(reinterpret_cast<const char*>(s->view.materials + materials[k])) +
                    offsetof(wf::Material, albedo);
        WF_CUDA(cudaMemcpy(dst, rgb + 3 * size_t(k), 3 * sizeof(float), cudaMemcpyHostToDevice));
    }
    return WF_OK;
}

wf_status wf_scene_set_environment(wf_scene* s, const wf_environment* env) {
    if (!s) return fail(WF_ERR_INVALID_ARG, "null scene");
    if (!env) {
        WF_CUDA(cudaDeviceSynchronize());
        free_list(s->env_allocations);
        s->device_bytes -= s->env_bytes;
        s->env_bytes = 0;
        s->view.env = Environment{};
        return WF_OK;
    }
    HostEnvironment map;
    if (wf_status e = build_environment(env, map)) return e;
    WF_CUDA(cudaDeviceSynchronize());
    free_list(s->env_allocations);
    s->device_bytes -= s->env_bytes;
    s->env_bytes = 0;
    Environment& ev = s->view.env;
    ev = Environment{};
    cudaError_t e = cudaSuccess;
    auto up = [&](auto** dst, const auto& vec) {
        if (e == cudaSuccess) e = upload(s, s->env_allocations, s->env_bytes, dst, vec);
    };
    up(&ev.pixels, map.pixels);
    up(&ev.probabilities, map.probabilities);
    up(&ev.alias, map.alias);
    up(&ev.row_solid_angle, map.row_solid_angle);
    if (e != cudaSuccess) {
        free_list(s->env_allocations);
        ev = Environment{};
        return cuda_fail(e, "environment upload");
    }
    s->device_bytes += s->env_bytes;
    ev.width = map.width;
    ev.height = map.height;
    ev.intensity = map.intensity;
    ev.rotation = map.rotation;
    ev.cos_rot = wfm::cosf(map.rotation);
    ev.sin_rot = wfm::sinf(map.rotation);
    ev.cos_neg = wfm::cosf(-map.rotation);
    ev.sin_neg = wfm::sinf(-map.rotation);
    ev.present = 1;
    ev.sampling = map.intensity > 0.0f ? 1u : 0u;
    return WF_OK;
}

wf_status wf_scene_destroy(wf_scene* s) {
    if (!s) return WF_OK;
    cudaDeviceSynchronize();
    free_list(s->allocations);
    free_list(s->env_allocations);
    delete s;
    return WF_OK;
}

wf_status wf_bvh_build(uint32_t builder, const float* boxes, uint32_t count, uint32_t* nodes,
                       double* milliseconds) {
    if ((count && !boxes) || (count && !nodes)) return fail(WF_ERR_INVALID_ARG, "null boxes or nodes");
    if (builder != WF_BVH_HOST_SAH && builder != WF_BVH_GPU_PLOC)
        return fail(WF_ERR_INVALID_ARG, "unknown BVH builder %u", builder);
    std::vector<BvhBox> prims(count);
    for (uint32_t i = 0; i < count; ++i)
        for (int a = 0; a < 3; ++a) {
            prims[i].lo[a] = boxes[6 * size_t(i) + a];
            prims[i].hi[a] = boxes[6 * size_t(i) + 3 + a];
        }
    std::vector<BvhBinaryNode> out;
    auto t0 = std::chrono::steady_clock::now();
    if (builder == WF_BVH_GPU_PLOC) {
        char why[256] = {0};
        if (!build_binary_bvh_gpu(prims.data(), count, out, 1 << 30, why, sizeof(why)))
            return fail(WF_ERR_CUDA, "GPU BVH build failed: %s", why);
    } else {
        build_binary_bvh(prims.data(), count, out, 0);
    }
    if (milliseconds) *milliseconds = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    static_assert(sizeof(BvhBinaryNode) == 8 * sizeof(uint32_t), "node record is 8 words");
    if (!out.empty()) std::memcpy(nodes, out.data(), sizeof(BvhBinaryNode) * out.size());
    return WF_OK;
}

wf_status wf_scene_get_info(const wf_scene* s, wf_scene_info* info) {
    if (!s || !info) return fail(WF_ERR_INVALID_ARG, "null argument");
    info->light_count = s->light_count;
    info->tlas_leaf_count = s->tlas_leaf_count;
    info->blas_count = s->blas_count;
    info->material_count = s->material_count;
    info->device_bytes = s->device_bytes;
    info->build_seconds = s->build_seconds;
    info->gpu_bvh_builds = s->gpu_bvh_builds;
    info->bvh_build_ms = float(s->bvh_build_ms);
    return WF_OK;
}

wf_status wf_trace_closest(const wf_scene* s, const wf_ray* rays, uint32_t count, wf_hit* hits, void* stream) {
    if (!s || (count && (!rays || !hits))) return fail(WF_ERR_INVALID_ARG, "null argument");
    return trace_closest_batch(s, rays, count, hits, static_cast<cudaStream_t>(stream));
}

wf_status wf_trace_any(const wf_scene* s, const wf_ray* rays, const float* max_distance, uint32_t count,
                       uint8_t* occluded, void* stream) {
    if (!s || (count && (!rays || !max_distance || !occluded))) return fail(WF_ERR_INVALID_ARG, "null argument");
    return trace_any_batch(s, rays, max_distance, count, occluded, static_cast<cudaStream_t>(stream));
}

wf_status wf_frame_guides(const wf_scene* s, const wf_camera* camera, const wf_camera* previous, uint32_t width,
                          uint32_t height, uint32_t x, uint32_t y, uint32_t w, uint32_t h, wf_frame_guide* guides,
                          void* stream) {
    if (!s || !camera || (uint64_t(w) * h && !guides)) return fail(WF_ERR_INVALID_ARG, "null argument");
    if (!width || !height || uint64_t(x) + w > width || uint64_t(y) + h > height)
        return fail(WF_ERR_INVALID_ARG, "tile (%u, %u, %u, %u) is outside the %u x %u image", x, y, w, h, width,
                    height);
    return frame_guides(s, camera, previous, width, height, x, y, w, h, guides, static_cast<cudaStream_t>(stream));
}

wf_status wf_renderer_create(const wf_scene* scene, const wf_camera* camera, const wf_render_config* config,
                             void* stream, wf_renderer** out) {
    return renderer_create(scene, camera, config, stream, out);
}

wf_status wf_renderer_destroy(wf_renderer* r) { return renderer_destroy(r); }

wf_status wf_render(wf_renderer* r, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_start,
                    uint32_t sample_count, uint32_t clear_tile) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    return renderer_render(r, x, y, w, h, sample_start, sample_count, clear_tile);
}

wf_status wf_render_frame(wf_renderer* r, uint32_t sample_count) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    return renderer_render_frame(r, sample_count);
}

wf_status wf_renderer_autotune(const wf_scene* scene, const wf_camera* camera, const wf_render_config* base,
                               const wf_tune_space* space, void* stream, wf_render_config* best, float* times_ms,
                               uint32_t times_capacity, uint32_t* evaluated) {
    if (!scene || !camera || !base || !space || !best) return fail(WF_ERR_INVALID_ARG, "null argument");
    auto values = [](const uint32_t* list, uint32_t count, uint32_t keep) {
        std::vector<uint32_t> v;
        for (uint32_t i = 0; list && i < count; ++i) v.push_back(list[i]);
        if (v.empty()) v.push_back(keep);
        return v;
    };
    std::vector<uint32_t> modes = values(space->modes, space->mode_count, base->mode);
    std::vector<uint32_t> blocks = values(space->block_sizes, space->block_size_count, base->block_size);
    std::vector<uint32_t> refills =
        values(space->refill_thresholds, space->refill_threshold_count, base->refill_threshold);
    std::vector<uint32_t> tiles = values(space->tile_sizes, space->tile_size_count,
                                         base->tile_width == base->tile_height ? base->tile_width : 0u);
    uint32_t samples = space->samples ? space->samples : 1u;
    uint32_t count = 0;
    float best_ms = 0.0f;
    bool have_best = false;
    for (uint32_t mode : modes) {
        // the mode's own settings: (setting, fused-kernel chunk) pairs
        std::vector<std::pair<uint32_t, uint32_t>> own;
        if (mode == WF_MODE_GRAPH) {  // (concurrent tiles, samples per wave)
            for (uint32_t v : values(space->concurrent_tiles, space->concurrent_tiles_count, base->concurrent_tiles))
                for (uint32_t w :
                     values(space->samples_per_waves, space->samples_per_wave_count, base->samples_per_wave))
                    own.push_back({v, w});
        } else if (mode == WF_MODE_STREAM) {
            for (uint32_t v :
                 values(space->regenerate_percents, space->regenerate_percent_count, base->regenerate_percent))
                own.push_back({v, base->chunk});
        } else {
            for (uint32_t k :
                 values(space->persistent_stages, space->persistent_stage_count, base->persistent_stages)) {
                if (k == WF_PERSISTENT_STAGED) {
                    own.push_back({k, base->chunk});
                    continue;
                }
                for (uint32_t chunk : values(space->chunks, space->chunk_count, base->chunk)) own.push_back({k, chunk});
            }
        }
        for (uint32_t block : blocks)
            for (uint32_t refill : refills)
                for (uint32_t tile : tiles)
                    for (const auto& setting : own) {
                        wf_render_config c = *base;
                        c.mode = mode;
                        c.block_size = block;
                        c.refill_threshold = refill;
                        c.tile_width = c.tile_height = tile;
                        if (mode == WF_MODE_GRAPH) {
                            c.concurrent_tiles = setting.first;
                            c.samples_per_wave = setting.second;
                        } else if (mode == WF_MODE_STREAM) {
                            c.regenerate_percent = setting.first;
                        } else {
                            c.persistent_stages = setting.first;
                            c.chunk = setting.second;
                        }
                        wf_renderer* r = nullptr;
                        if (wf_status e = renderer_create(scene, camera, &c, stream, &r)) {
                            if (e != WF_ERR_OOM) return e;
                            // a candidate whose queues do not fit (a large wave) is skipped
                            cudaGetLastError();
                            if (times_ms && count < times_capacity) times_ms[count] = INFINITY;
                            ++count;
                            continue;
                        }
                        cudaEvent_t e0 = nullptr, e1 = nullptr;
                        float ms = 0.0f;
                        wf_status st = renderer_render_frame(r, samples);
                        cudaError_t err = cudaSuccess;
                        if (st == WF_OK) err = cudaEventCreate(&e0);
                        if (st == WF_OK && err == cudaSuccess) err = cudaEventCreate(&e1);
                        if (st == WF_OK && err == cudaSuccess) err = cudaEventRecord(e0, r->stream);
                        if (st == WF_OK && err == cudaSuccess) st = renderer_render_frame(r, samples);
                        if (st == WF_OK && err == cudaSuccess) err = cudaEventRecord(e1, r->stream);
                        if (st == WF_OK && err == cudaSuccess) err = cudaEventSynchronize(e1);
                        if (st == WF_OK && err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
                        if (st == WF_OK && err == cudaSuccess) st = wf_synchronize(r);
                        if (e0) cudaEventDestroy(e0);
                        if (e1) cudaEventDestroy(e1);
                        renderer_destroy(r);
                        if (st != WF_OK) return st;
                        if (err != cudaSuccess) return cuda_fail(err, "autotune timing");
                        if (times_ms && count < times_capacity) times_ms[count] = ms;
                        if (!have_best || ms < best_ms) {
                            best_ms = ms;
                            *best = c;
                            have_best = true;
                        }
                        ++count;
                    }
    }
    if (evaluated) *evaluated = count;
    if (!have_best) return fail(WF_ERR_OOM, "no autotune candidate fits in device memory");
    return WF_OK;
}

wf_status wf_profile_sample(wf_renderer* r, wf_kernel_profile* profile) {
    if (!r || !profile) return fail(WF_ERR_INVALID_ARG, "null argument");
    return renderer_profile(r, profile);
}

wf_status wf_framebuffer_reset(wf_renderer* r) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    size_t pixels = size_t(r->config.width) * r->config.height;
    WF_CUDA(cudaMemsetAsync(r->framebuffer, 0, sizeof(float) * 3 * pixels, r->stream));
    wf_renderer* parts[2];
    for (int i = 0, n = renderer_parts(r, parts); i < n; ++i)
        WF_CUDA(cudaMemsetAsync(&parts[i]->counters->sample_index, 0, sizeof(uint32_t), parts[i]->stream));
    return WF_OK;
}

wf_status wf_set_sample_index(wf_renderer* r, uint32_t sample_index) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    wf_renderer* parts[2];
    for (int i = 0, n = renderer_parts(r, parts); i < n; ++i) {
        WF_CUDA(cudaMemcpyAsync(&parts[i]->counters->sample_index, &sample_index, sizeof(uint32_t),
                                cudaMemcpyHostToDevice, parts[i]->stream));
        WF_CUDA(cudaStreamSynchronize(parts[i]->stream));
    }
    return WF_OK;
}

wf_status wf_get_sample_index(wf_renderer* r, uint32_t* sample_index) {
    if (!r || !sample_index) return fail(WF_ERR_INVALID_ARG, "null argument");
    WF_CUDA(cudaMemcpyAsync(sample_index, &r->counters->sample_index, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            r->stream));
    WF_CUDA(cudaStreamSynchronize(r->stream));
    return WF_OK;
}

wf_status wf_synchronize(wf_renderer* r) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    uint32_t flags[2] = {0, 0};
    if (r->copy_stream) WF_CUDA(cudaStreamSynchronize(r->copy_stream));
    wf_renderer* parts[2];
    for (int i = 0, n = renderer_parts(r, parts); i < n; ++i) {
        WF_CUDA(cudaStreamSynchronize(parts[i]->stream));
        uint32_t f[2] = {0, 0};
        WF_CUDA(cudaMemcpy(&f[0], &parts[i]->counters->overflow, sizeof(uint32_t), cudaMemcpyDeviceToHost));
        WF_CUDA(cudaMemcpy(&f[1], &parts[i]->counters->error, sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (f[0] || f[1]) {  // reported once: the next render starts clean
            WF_CUDA(cudaMemset(&parts[i]->counters->overflow, 0, sizeof(uint32_t)));
            WF_CUDA(cudaMemset(&parts[i]->counters->error, 0, sizeof(uint32_t)));
        }
        flags[0] |= f[0];
        flags[1] = flags[1] ? flags[1] : f[1];
    }
    if (flags[1] == wf::kErrorStreamBound)
        return fail(WF_ERR_TIMEOUT, "streaming loop exceeded samples x max_depth iterations");
    if (flags[1]) return fail(WF_ERR_TIMEOUT, "persistent kernel grid barrier timed out");
    if (flags[0]) return fail(WF_ERR_CAPACITY, "shadow queue or term buffer overflow (flags %u)", flags[0]);
    return WF_OK;
}

wf_status wf_renderer_set_watchdog(wf_renderer* r, uint64_t barrier_cycles, uint32_t loop_iterations) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    wf_renderer* parts[2];
    for (int i = 0, n = renderer_parts(r, parts); i < n; ++i) {
        Counters* c = parts[i]->counters;
        unsigned long long cycles = barrier_cycles;
        WF_CUDA(cudaMemcpyAsync(&c->barrier_limit, &cycles, sizeof(cycles), cudaMemcpyHostToDevice,
                                parts[i]->stream));
        WF_CUDA(cudaMemcpyAsync(&c->stream_limit, &loop_iterations, sizeof(loop_iterations), cudaMemcpyHostToDevice,
                                parts[i]->stream));
        WF_CUDA(cudaStreamSynchronize(parts[i]->stream));  // the host values are on this stack
    }
    return WF_OK;
}

wf_status wf_framebuffer_download(wf_renderer* r, uint32_t x, uint32_t y, uint32_t w, uint32_t h, float* rgb) {
    if (!r || !rgb) return fail(WF_ERR_INVALID_ARG, "null argument");
    const wf_render_config& c = r->config;
    if (w == 0 || h == 0 || x >= c.width || y >= c.height || w > c.width - x || h > c.height - y)
        return fail(WF_ERR_INVALID_ARG, "download region outside the framebuffer");
    WF_CUDA(cudaMemcpy2DAsync(rgb, size_t(w) * 12, r->framebuffer + (size_t(y) * c.width + x) * 3,
                              size_t(c.width) * 12, size_t(w) * 12, h, cudaMemcpyDeviceToHost, r->stream));
    return wf_synchronize(r);
}

wf_status wf_framebuffer_download_async(wf_renderer* r, uint32_t x, uint32_t y, uint32_t w, uint32_t h,
                                        float* rgb) {
    if (!r || !rgb) return fail(WF_ERR_INVALID_ARG, "null argument");
    const wf_render_config& c = r->config;
    if (w == 0 || h == 0 || x >= c.width || y >= c.height || w > c.width - x || h > c.height - y)
        return fail(WF_ERR_INVALID_ARG, "download region outside the framebuffer");
    if (!r->copy_stream) {
        size_t full = size_t(c.width) * c.height * 3 * sizeof(float);
        for (int k = 0; k < 2; ++k) {  // a call that failed half-way left some of these
            if (!r->snapshot[k]) {
                void* p = nullptr;
                cudaError_t e = device_alloc(&p, full);
                if (e != cudaSuccess) return cuda_fail(e, "framebuffer snapshot");
                r->allocations.push_back(p);
                r->device_bytes += full;
                r->snapshot[k] = static_cast<float*>(p);
            }
            if (!r->snapshot_ready[k]) WF_CUDA(cudaEventCreateWithFlags(&r->snapshot_ready[k], cudaEventDisableTiming));
            if (!r->copy_done[k]) WF_CUDA(cudaEventCreateWithFlags(&r->copy_done[k], cudaEventDisableTiming));
        }
        WF_CUDA(cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking));
    }
    uint32_t k = r->next_snapshot;
    r->next_snapshot ^= 1u;
    // the snapshot's previous copy must have left before it is overwritten
    WF_CUDA(cudaStreamWaitEvent(r->stream, r->copy_done[k], 0));
    WF_CUDA(cudaMemcpy2DAsync(r->snapshot[k], size_t(w) * 12, r->framebuffer + (size_t(y) * c.width + x) * 3,
                              size_t(c.width) * 12, size_t(w) * 12, h, cudaMemcpyDeviceToDevice, r->stream));
    WF_CUDA(cudaEventRecord(r->snapshot_ready[k], r->stream));
    WF_CUDA(cudaStreamWaitEvent(r->copy_stream, r->snapshot_ready[k], 0));
    WF_CUDA(cudaMemcpyAsync(rgb, r->snapshot[k], size_t(w) * h * 12, cudaMemcpyDeviceToHost, r->copy_stream));
    WF_CUDA(cudaEventRecord(r->copy_done[k], r->copy_stream));
    return WF_OK;
}

wf_status wf_framebuffer_download_wait(wf_renderer* r) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    if (!r->copy_stream) return WF_OK;
    for (int k = 0; k < 2; ++k) WF_CUDA(cudaStreamWaitEvent(r->stream, r->copy_done[k], 0));
    WF_CUDA(cudaStreamSynchronize(r->copy_stream));
    return WF_OK;
}

wf_status wf_framebuffer_device(wf_renderer* r, float** rgb) {
    if (!r || !rgb) return fail(WF_ERR_INVALID_ARG, "null argument");
    *rgb = r->framebuffer;
    return WF_OK;
}

wf_status wf_queue_counts(wf_renderer* r, uint32_t* counts, uint32_t n) {
    if (!r || !counts) return fail(WF_ERR_INVALID_ARG, "null argument");
    uint32_t m = std::min(n, r->config.max_depth);
    std::vector<uint32_t> part(m);
    std::fill(counts, counts + m, 0u);
    wf_renderer* parts[2];
    for (int i = 0, k = renderer_parts(r, parts); i < k; ++i) {  // the parts that rendered the last tile
        if (!(r->last_tile_parts & (1u << i))) continue;
        WF_CUDA(cudaMemcpyAsync(part.data(), parts[i]->counters->profile, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost,
                                parts[i]->stream));
        WF_CUDA(cudaStreamSynchronize(parts[i]->stream));
        for (uint32_t b = 0; b < m; ++b) counts[b] += part[b];
    }
    return WF_OK;
}

wf_status wf_render_stats_get(wf_renderer* r, wf_render_stats* stats, uint32_t reset) {
    if (!r || !stats) return fail(WF_ERR_INVALID_ARG, "null argument");
    std::memset(stats, 0, sizeof(*stats));
    wf_renderer* parts[2];
    for (int i = 0, n = renderer_parts(r, parts); i < n; ++i) {
        unsigned long long v[4];
        WF_CUDA(cudaMemcpyAsync(v, &parts[i]->counters->extension_rays, sizeof(v), cudaMemcpyDeviceToHost,
                                parts[i]->stream));
        WF_CUDA(cudaStreamSynchronize(parts[i]->stream));
        stats->extension_rays += v[0];
        stats->shadow_rays += v[1];
        stats->paths += v[2];
        stats->kernel_launches += v[3];
        if (reset) {
            WF_CUDA(cudaMemsetAsync(&parts[i]->counters->extension_rays, 0, sizeof(v), parts[i]->stream));
            WF_CUDA(cudaStreamSynchronize(parts[i]->stream));
        }
    }
    return WF_OK;
}

wf_status wf_photon_stats(wf_renderer* r, uint32_t* stored, uint32_t* emitted) {
    if (!r || !stored || !emitted) return fail(WF_ERR_INVALID_ARG, "null argument");
    *stored = r->photons_stored;
    *emitted = r->photons_emitted;
    return WF_OK;
}

wf_status wf_photons_download(wf_renderer* r, float* records, uint32_t count) {
    if (!r || !records) return fail(WF_ERR_INVALID_ARG, "null argument");
    if (!r->photon_raw || count > r->photons_emitted) return fail(WF_ERR_STATE, "no photon map of that size");
    std::vector<float4> raw(size_t(count) * 4);
    WF_CUDA(cudaMemcpyAsync(raw.data(), r->photon_raw, sizeof(float4) * raw.size(), cudaMemcpyDeviceToHost, r->stream));
    WF_CUDA(cudaStreamSynchronize(r->stream));
    for (uint32_t i = 0; i < count; ++i) {
        const float4* p = &raw[4 * size_t(i)];
        float* o = records + 8 * size_t(i);
        o[0] = p[0].x; o[1] = p[0].y; o[2] = p[0].z;
        o[3] = p[1].x; o[4] = p[1].y; o[5] = p[1].z;
        o[6] = p[2].x + p[2].y + p[2].z;
        o[7] = p[0].w;
    }
    return WF_OK;
}

wf_status wf_checkpoint_save(wf_renderer* r, const char* path, uint64_t fingerprint) {
    if (!r || !path) return fail(WF_ERR_INVALID_ARG, "null argument");
    size_t pixels = size_t(r->config.width) * r->config.height;
    std::vector<float> rgb(pixels * 3);
    uint32_t sample = 0;
    WF_CUDA(cudaMemcpyAsync(rgb.data(), r->framebuffer, sizeof(float) * rgb.size(), cudaMemcpyDeviceToHost, r->stream));
    WF_CUDA(cudaMemcpyAsync(&sample, &r->counters->sample_index, sizeof(uint32_t), cudaMemcpyDeviceToHost, r->stream));
    WF_CUDA(cudaStreamSynchronize(r->stream));
    return write_checkpoint(path, rgb.data(), r->config.width, r->config.height, sample, fingerprint);
}

wf_status wf_checkpoint_enqueue(wf_renderer* r, const char* path, uint64_t fingerprint, uint32_t* queued) {
    if (!r || !path || !queued) return fail(WF_ERR_INVALID_ARG, "null argument");
    *queued = 0;
    size_t pixels = size_t(r->config.width) * r->config.height;
    if (r->slots.empty()) {
        for (int i = 0; i < 3; ++i) {
            auto slot = std::make_unique<AsyncCheckpointSlot>();
            WF_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&slot->pixels), sizeof(float) * 3 * pixels + 16,
                                  cudaHostAllocDefault));
            WF_CUDA(cudaEventCreateWithFlags(&slot->copied, cudaEventDisableTiming));
            r->slots.push_back(std::move(slot));
        }
    }
    for (auto& sp : r->slots) {
        AsyncCheckpointSlot& slot = *sp;
        bool expected = false;
        if (!slot.busy.compare_exchange_strong(expected, true)) continue;
        if (slot.writer.joinable()) slot.writer.join();
        // The sample index travels with the pixels (last float slot).
        WF_CUDA(cudaMemcpyAsync(slot.pixels, r->framebuffer, sizeof(float) * 3 * pixels, cudaMemcpyDeviceToHost,
                                r->stream));
        WF_CUDA(cudaMemcpyAsync(slot.pixels + 3 * pixels, &r->counters->sample_index, sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, r->stream));
        WF_CUDA(cudaEventRecord(slot.copied, r->stream));
        std::string file = path;
        uint32_t width = r->config.width, height = r->config.height;
        wf_renderer* rr = r;
        slot.writer = std::thread([rr, &slot, file, fingerprint, width, height, pixels] {
            cudaEventSynchronize(slot.copied);
            uint32_t sample;
            std::memcpy(&sample, slot.pixels + 3 * pixels, 4);
            {
                std::lock_guard<std::mutex> lock(rr->write_mutex);
                if (sample >= rr->latest_written) {
                    write_checkpoint(file.c_str(), slot.pixels, width, height, sample, fingerprint);
                    rr->latest_written = sample;
                }
            }
            slot.busy.store(false);
        });
        *queued = 1;
        return WF_OK;
    }
    return WF_OK;
}

wf_status wf_checkpoint_flush(wf_renderer* r) {
    if (!r) return fail(WF_ERR_INVALID_ARG, "null renderer");
    for (auto& slot : r->slots)
        if (slot->writer.joinable()) slot->writer.join();
    return WF_OK;
}

wf_status wf_checkpoint_load(wf_renderer* r, const char* path, uint64_t fingerprint, uint32_t* sample_index) {
    if (!r || !path || !sample_index) return fail(WF_ERR_INVALID_ARG, "null argument");
    std::ifstream in(path, std::ios::binary);
    if (!in) return fail(WF_ERR_IO, "Could not open checkpoint: %s", path);
    CheckpointHeader header{};
    in.read(reinterpret_cast<char*>(&header), sizeof(header));
    if (!in) return fail(WF_ERR_FORMAT, "Checkpoint is truncated or unreadable: %s", path);
    if (std::memcmp(header.magic, kMagic, 8) != 0 || header.version != kCheckpointVersion)
        return fail(WF_ERR_FORMAT, "Unsupported checkpoint format: %s", path);
    if (header.width != r->config.width || header.height != r->config.height)
        return fail(WF_ERR_FORMAT, "Checkpoint resolution does not match the current render: %s", path);
    if (header.fingerprint != fingerprint)
        return fail(WF_ERR_FINGERPRINT, "Checkpoint scene/config fingerprint does not match the current render: %s", path);
    size_t pixels = size_t(header.width) * header.height;
    std::vector<float> rgb(pixels * 3);
    in.read(reinterpret_cast<char*>(rgb.data()), std::streamsize(sizeof(float) * rgb.size()));
    if (!in) return fail(WF_ERR_FORMAT, "Checkpoint is truncated or unreadable: %s", path);
    WF_CUDA(cudaMemcpyAsync(r->framebuffer, rgb.data(), sizeof(float) * rgb.size(), cudaMemcpyHostToDevice, r->stream));
    WF_CUDA(cudaMemcpyAsync(&r->counters->sample_index, &header.sample_index, sizeof(uint32_t), cudaMemcpyHostToDevice,
                            r->stream));
    WF_CUDA(cudaStreamSynchronize(r->stream));
    if (r->twin) {
        WF_CUDA(cudaMemcpyAsync(&r->twin->counters->sample_index, &header.sample_index, sizeof(uint32_t),
                                cudaMemcpyHostToDevice, r->twin->stream));
        WF_CUDA(cudaStreamSynchronize(r->twin->stream));
    }
    *sample_index = header.sample_index;
    return WF_OK;
}

uint64_t wf_fnv1a64(const void* data, size_t size, uint64_t seed) {
    uint64_t h = seed ? seed : 1469598103934665603ull;
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < size; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

}  // extern "C"
