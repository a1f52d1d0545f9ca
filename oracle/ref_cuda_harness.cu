// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into or called by the
// product.  Only bench.py's --reference-cuda measurement and the script beside
// it (oracle/ref_cuda_bench.py) load the library built from this file
// (oracle/_ref/libwfref_cuda.so).
//
// The reference's own CUDA renderer on this GPU: its sources (src/scene/scene.cu,
// src/renderer/renderer.cu, render_driver.cu, render_task.cu, ...) are
// compiled unmodified for sm_100a by oracle/Makefile (target `cuda`), with the
// reference's separable compilation and nvcc's default floating-point flags.
// This file only converts the C-ABI scene description into the reference's
// HostScene (ref_scene_convert.h), calls the reference's uploadScene and
// uploadEnvironmentMap, and renders whole-frame tasks through the reference's
// RenderTaskRenderer::render (src/renderer/render_task.cu:26-114), the call a
// distributed worker makes: clear the tile, render the sample range with the
// captured graph or the persistent kernel, download the radiance.
//
// NexusBVH is absent, so the BVH2 builds that scene.cu asks for are answered
// here with the project's binned-SAH builder (the same trees the host build of
// the reference and the B200 renderer traverse), built on the host and
// uploaded (shim_cuda/NXB/BVH.h).
// Standard headers first: the access override below must not reach them.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "config.hpp"
#include "renderer/image_output.hpp"
// The photon map of a caustic render is built here with the reference's
// public kernels (emitPhotons / tracePhotons / buildPhotonGrid,
// include/renderer/renderer.cuh:34-41) and handed to the driver's resources
// before its graph is captured, in place of RenderDriver::buildPhotonMap,
// whose grid has fixed Cornell-box bounds (render_driver.cu:211-213) and runs
// only for the Cornell family of presets (render_driver.cu:181-182).  That
// needs the driver's private members, opened for this file only.
#define private public
#include "renderer/render_driver.cuh"
#undef private
#include "renderer/render_fingerprint.hpp"
#include "renderer/render_task.cuh"
#include "renderer/renderer.cuh"
#include "scene/environment.hpp"
#include "scene/scene_host.hpp"

#include "../wavefront-path-tracer_b200/csrc/bvh_build.h"
#include "ref_scene_convert.h"

// ------------------------------------------------------------ NXB builder
namespace {
NXB::BVH2 build_nexus(std::vector<wf::BvhBox>& boxes) {
    std::vector<wf::BvhBinaryNode> nodes;
    wf::build_binary_bvh(boxes.data(), uint32_t(boxes.size()), nodes, 0);
    std::vector<NXB::BVH2::Node> host(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        const wf::BvhBinaryNode& n = nodes[i];
        host[i].bounds = NXB::AABB(make_float3(n.box.lo[0], n.box.lo[1], n.box.lo[2]),
                                   make_float3(n.box.hi[0], n.box.hi[1], n.box.hi[2]));
        host[i].leftChild = n.left;
        host[i].rightChild = n.right;
    }
    NXB::BVH2 bvh;
    bvh.nodes_ = NXB::detail::device_copy(host.data(), host.size());
    bvh.nodeCount_ = uint32_t(host.size());
    bvh.primCount_ = uint32_t(boxes.size());
    if (!host.empty()) bvh.bounds_ = host.back().bounds;  // the root is the last node
    return bvh;
}

void download(void* dst, const void* src, size_t bytes) {
    if (bytes && cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("NXB shim: cudaMemcpy from the device failed");
}
}  // namespace

namespace NXB {
BVH2 BuildBVH2(const Triangle* triangles, uint32_t count, BuildConfig, BVHBuildMetrics*) {
    static_assert(sizeof(Triangle) == 9 * sizeof(float), "NXB::Triangle is three float3");
    std::vector<float> v(size_t(count) * 9);
    download(v.data(), triangles, sizeof(Triangle) * size_t(count));
    std::vector<wf::BvhBox> boxes(count);
    for (uint32_t i = 0; i < count; ++i) {
        const float* t = &v[size_t(i) * 9];
        for (int a = 0; a < 3; ++a) {
            boxes[i].lo[a] = std::min(std::min(t[a], t[3 + a]), t[6 + a]);
            boxes[i].hi[a] = std::max(std::max(t[a], t[3 + a]), t[6 + a]);
        }
    }
    return build_nexus(boxes);
}
BVH2 BuildBVH2(const AABB* aabbs, uint32_t count, BuildConfig, BVHBuildMetrics*) {
    std::vector<AABB> host(count);
    download(host.data(), aabbs, sizeof(AABB) * size_t(count));
    std::vector<wf::BvhBox> boxes(count);
    for (uint32_t i = 0; i < count; ++i)
        boxes[i] = wf::BvhBox{{host[i].bMin.x, host[i].bMin.y, host[i].bMin.z},
                              {host[i].bMax.x, host[i].bMax.y, host[i].bMax.z}};
    return build_nexus(boxes);
}
BVH8 BuildBVH8(const Triangle*, uint32_t, BuildConfig, BVHBuildMetrics*) {
    throw std::runtime_error("BVH8 is not provided by the NexusBVH shim");
}
}  // namespace NXB

// RenderDriver::writeFinalImage (render_driver.cu:403-418) is reached only
// from RenderDriver::run, which this harness does not call; the PPM writer
// and its SHA-256 digest (image_output.cpp, OpenSSL) are not linked.
std::string sha256Framebuffer(const std::vector<Vec3>&) { return std::string(); }
void writePpm(const char*, const std::vector<Vec3>&, uint32_t, uint32_t) {}

namespace {
struct CudaRefScene {
    DeviceScene device;
    bool probe = false;
    uint32_t original_material_count = 0;
};

// The reference's traceRayExternal (device_traversal.cuh:1196) over a batch
// of rays, one per thread.
__global__ void k_ref_trace(Scene scene, const wf_ray* rays, uint32_t count, TraceResult* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Ray ray(Vec3(rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]),
            Vec3(rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]));
    out[i] = traceRayExternal(ray, scene);
}
}  // namespace

namespace {
#define WFCUDA_CHECK(call)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// RenderDriver::buildPhotonMap (render_driver.cu:180-234) with the grid
// bounds taken from the stored photons instead of the Cornell constants:
// the bounding box of the valid photons, with a degenerate axis given unit
// extent -- the bounds the B200 renderer derives when its config's grid
// minimum equals its maximum.  Explicit bounds (min != max) are used as
// given.  Returns the build's wall time in milliseconds.
double build_photon_map(RenderDriver& driver, const wf_render_config* c) {
    auto t0 = std::chrono::steady_clock::now();
    RenderResources& res = driver.resources_;
    const Scene& scene = driver.deviceScene_.scene;
    uint32_t n = c->photon_count;
    WFCUDA_CHECK(cudaDeviceSetLimit(cudaLimitStackSize, 16 * 1024));  // as buildPhotonMap sets it
    WFCUDA_CHECK(cudaMalloc(&res.devicePhotons, sizeof(Photon) * n));
    WFCUDA_CHECK(cudaMalloc(&res.devicePhotonMaterialHitCounts, sizeof(uint32_t) * 3));
    WFCUDA_CHECK(cudaMemset(res.devicePhotonMaterialHitCounts, 0, sizeof(uint32_t) * 3));
    WFCUDA_CHECK(cudaMemset(res.devicePhotons, 0, sizeof(Photon) * n));
    res.photonQueue.items = res.devicePhotons;
    res.photonQueue.capacity = n;
    uint32_t block = driver.config_.blockSize;
    uint32_t blocks = (n + block - 1) / block;
    emitPhotons<<<blocks, block>>>(res.photonQueue, scene, n, c->photon_seed, RngStrategy(c->rng), c->spectral != 0);
    WFCUDA_CHECK(cudaGetLastError());
    tracePhotons<<<blocks, block>>>(res.photonQueue, scene, n, c->photon_max_depth, res.devicePhotonMaterialHitCounts);
    WFCUDA_CHECK(cudaGetLastError());
    WFCUDA_CHECK(cudaDeviceSynchronize());
    PhotonGrid grid{};
    grid.photons = res.devicePhotons;
    grid.resolution = c->photon_grid_resolution ? c->photon_grid_resolution : 64;
    bool derive = c->photon_grid_min[0] == c->photon_grid_max[0] && c->photon_grid_min[1] == c->photon_grid_max[1] &&
                  c->photon_grid_min[2] == c->photon_grid_max[2];
    if (derive) {
        std::vector<Photon> host(n);
        WFCUDA_CHECK(cudaMemcpy(host.data(), res.devicePhotons, sizeof(Photon) * n, cudaMemcpyDeviceToHost));
        float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        bool any = false;
        for (const Photon& p : host) {
            if (!p.valid) continue;
            float v[3] = {p.position.x, p.position.y, p.position.z};
            for (int a = 0; a < 3; ++a) {
                lo[a] = any ? std::min(lo[a], v[a]) : v[a];
                hi[a] = any ? std::max(hi[a], v[a]) : v[a];
            }
            any = true;
        }
        if (!any) {
            for (int a = 0; a < 3; ++a) lo[a] = -1.0f, hi[a] = 1.0f;
        }
        for (int a = 0; a < 3; ++a)
            if (!(hi[a] > lo[a])) hi[a] = lo[a] + 1.0f;
        grid.minimum = Vec3(lo[0], lo[1], lo[2]);
        grid.maximum = Vec3(hi[0], hi[1], hi[2]);
    } else {
        grid.minimum = Vec3(c->photon_grid_min[0], c->photon_grid_min[1], c->photon_grid_min[2]);
        grid.maximum = Vec3(c->photon_grid_max[0], c->photon_grid_max[1], c->photon_grid_max[2]);
    }
    uint32_t cells = grid.resolution * grid.resolution * grid.resolution;
    WFCUDA_CHECK(cudaMalloc(&grid.heads, sizeof(uint32_t) * cells));
    WFCUDA_CHECK(cudaMalloc(&grid.next, sizeof(uint32_t) * n));
    WFCUDA_CHECK(cudaMemset(grid.heads, 0xff, sizeof(uint32_t) * cells));
    WFCUDA_CHECK(cudaMemset(grid.next, 0xff, sizeof(uint32_t) * n));
    buildPhotonGrid<<<blocks, block>>>(res.photonQueue, grid, n);
    WFCUDA_CHECK(cudaGetLastError());
    WFCUDA_CHECK(cudaDeviceSynchronize());
    res.photonGrid = grid;  // released with the driver's resources
    res.shadingPhotonGrid = grid;
    if (!c->caustic_gather) res.shadingPhotonGrid.heads = nullptr;
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

namespace {
Camera reference_camera(const wf_camera* cam) {
    Camera camera;
    camera.position = wfref::v3(cam->position);
    camera.forward = wfref::v3(cam->forward);
    camera.right = wfref::v3(cam->right);
    camera.up = wfref::v3(cam->up);
    camera.verticalFov = cam->vertical_fov;
    camera.aspectRatio = cam->aspect_ratio;
    return camera;
}

// The reference's RenderConfig for a wf_render_config.  A config with a tile
// size renders tiled (the queues hold one tile), which keeps the launches of
// a small task small.
RenderConfig reference_config(const wf_render_config* c, int persistent, bool profile_queues) {
    RenderConfig config;
    config.width = c->width;
    config.height = c->height;
    config.maxDepth = c->max_depth;
    config.russianRouletteStartDepth = c->rr_start_depth;
    config.samplesPerPixel = 1u << 30;  // bounds the absolute sample ranges of tasks
    config.persistentWavefront = persistent != 0;
    config.indirectRadianceClamp = c->indirect_clamp;
    config.rngStrategy = RngStrategy(c->rng);
    config.blockSize = 256;
    if (c->tile_width && c->tile_height) {
        config.tiledRendering = true;
        config.tileWidth = c->tile_width;
        config.tileHeight = c->tile_height;
    }
    // The Demo preset is not a caustic preset, so prepare() builds no photon
    // map of its own; a caustic render gets the one build_photon_map makes.
    config.enableCaustics = c->caustics != 0;
    config.enableCausticGather = c->caustic_gather != 0;
    config.causticPhotonCount = c->caustics ? c->photon_count : config.causticPhotonCount;
    config.causticMaxDepth = c->photon_max_depth;
    config.causticGatherRadius = c->gather_radius;
    config.profileQueues = profile_queues;
    config.distributedRole = DistributedRole::Worker;  // no local checkpoint writer
    return config;
}
}  // namespace

extern "C" {

// probe != 0: the hit-identity probe copy of the scene (ref_scene_convert.h;
// instance lightOffset = index << 24), for wfcuda_trace.
void* wfcuda_scene_create_probe(const wf_scene_desc* d, const wf_environment* env, int probe) {
    try {
        HostScene h;
        wfref::host_scene_from_desc(d, probe != 0, h);
        auto r = std::make_unique<CudaRefScene>();
        r->probe = probe != 0;
        r->original_material_count = d->material_count;
        r->device = uploadScene(h);
        r->device.scene.ignoreDirectLightOcclusion = d->ignore_direct_light_occlusion != 0;
        wfref::apply_normal_map_settings(r->device.scene, d);
        if (probe && r->device.scene.instanceCount) {
            std::vector<MeshInstance> inst(r->device.scene.instanceCount);
            WFCUDA_CHECK(cudaMemcpy(inst.data(), r->device.instances, sizeof(MeshInstance) * inst.size(),
                                    cudaMemcpyDeviceToHost));
            for (uint32_t i = 0; i < inst.size(); ++i) inst[i].lightOffset = i << 24;
            WFCUDA_CHECK(cudaMemcpy(r->device.instances, inst.data(), sizeof(MeshInstance) * inst.size(),
                                    cudaMemcpyHostToDevice));
        }
        if (env && env->width && env->height) {
            HostEnvironment map;
            map.width = env->width;
            map.height = env->height;
            map.pixels.resize(size_t(env->width) * env->height);
            for (size_t i = 0; i < map.pixels.size(); ++i)
                map.pixels[i] = make_float4(env->rgba[4 * i], env->rgba[4 * i + 1], env->rgba[4 * i + 2],
                                            env->rgba[4 * i + 3]);
            buildEnvironmentDistribution(map);
            uploadEnvironmentMap(r->device, map, env->intensity, env->rotation_degrees);
        }
        if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
        return r.release();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfcuda_scene_create: %s\n", e.what());
        return nullptr;
    }
}

void* wfcuda_scene_create(const wf_scene_desc* d, const wf_environment* env) {
    return wfcuda_scene_create_probe(d, env, 0);
}

// Closest hits of `count` host rays with the reference's traversal on the
// GPU, as wf_hit records (the probe copy fills kind / primitive / instance
// from its identity codes, as oracle/ref_harness.cpp's wfref_trace does).
int wfcuda_trace(void* handle, const wf_ray* rays, uint32_t count, wf_hit* hits) {
    try {
        CudaRefScene* r = static_cast<CudaRefScene*>(handle);
        if (!r) return 1;
        if (count == 0) return 0;
        wf_ray* d_rays = nullptr;
        TraceResult* d_out = nullptr;
        WFCUDA_CHECK(cudaMalloc(&d_rays, sizeof(wf_ray) * count));
        WFCUDA_CHECK(cudaMalloc(&d_out, sizeof(TraceResult) * count));
        WFCUDA_CHECK(cudaMemcpy(d_rays, rays, sizeof(wf_ray) * count, cudaMemcpyHostToDevice));
        k_ref_trace<<<(count + 127) / 128, 128>>>(r->device.scene, d_rays, count, d_out);
        WFCUDA_CHECK(cudaGetLastError());
        std::vector<TraceResult> res(count);
        WFCUDA_CHECK(cudaMemcpy(res.data(), d_out, sizeof(TraceResult) * count, cudaMemcpyDeviceToHost));
        cudaFree(d_rays);
        cudaFree(d_out);
        for (uint32_t i = 0; i < count; ++i) {
            wf_hit& o = hits[i];
            std::memset(&o, 0, sizeof(o));
            o.instance = 0xffffffffu;
            o.primitive = 0xffffffffu;
            if (!res[i].didHit) {
                o.material = WF_NO_MATERIAL;
                o.light_index = 0xffffffffu;
                o.kind = WF_HIT_NONE;
                o.t = 1e30f;
                continue;
            }
            const Hit& h = res[i].hit;
            o.t = h.t;
            o.position[0] = h.position.x; o.position[1] = h.position.y; o.position[2] = h.position.z;
            o.geometric_normal[0] = h.geometricNormal.x;
            o.geometric_normal[1] = h.geometricNormal.y;
            o.geometric_normal[2] = h.geometricNormal.z;
            o.normal[0] = h.normal.x; o.normal[1] = h.normal.y; o.normal[2] = h.normal.z;
            o.material = h.material;
            o.light_index = h.lightIndex;
            o.kind = WF_HIT_NONE;
            if (r->probe) {
                if (h.material >= r->original_material_count) {
                    o.kind = WF_HIT_SPHERE;
                    o.primitive = h.material - r->original_material_count;
                } else if (h.lightIndex & 0x80000000u) {
                    o.kind = WF_HIT_TRIANGLE;
                    o.primitive = h.lightIndex & 0x3fffffffu;
                } else if (h.lightIndex & 0x40000000u) {
                    o.kind = WF_HIT_STATIC_TRIANGLE;
                    o.primitive = h.lightIndex & 0x3fffffffu;
                } else {
                    o.kind = WF_HIT_MESH;
                    o.instance = h.lightIndex >> 24;
                    o.primitive = h.lightIndex & 0xffffffu;
                }
            }
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfcuda_trace: %s\n", e.what());
        return 3;
    }
}

void wfcuda_scene_destroy(void* handle) {
    CudaRefScene* r = static_cast<CudaRefScene*>(handle);
    if (!r) return;
    destroyDeviceScene(r->device);
    delete r;
}


// Renders one warm-up task and then `steps` whole-frame tasks of `spp`
// samples each (absolute samples from sample_start on) through
// RenderTaskRenderer::render.  task_ms[i] is the wall time of task i, which
// covers the reference's own clear, launches, stream synchronisation and
// download; rgb (optional) receives the last task's unnormalised sums.
// With c->caustics the photon map is built first (build_photon_map above)
// and *photon_ms receives its wall time.  queue_counts (optional, max_depth
// entries) receives the reference's per-bounce queue sizes of the last task
// in persistent mode (its --profile-queues record, renderer.cu:89-90).
int wfcuda_render(void* handle, const wf_camera* cam, const wf_render_config* c, int persistent,
                  uint32_t sample_start, uint32_t spp, uint32_t steps, float* rgb, double* task_ms,
                  double* photon_ms, uint32_t* queue_counts) {
    try {
        CudaRefScene* r = static_cast<CudaRefScene*>(handle);
        if (!r || spp == 0) return 1;
        Camera camera = reference_camera(cam);
        RenderConfig config = reference_config(c, persistent, persistent && queue_counts != nullptr);
        SceneConfig scene_config;
        scene_config.preset = ScenePreset::Demo;
        RenderDriver driver(r->device, camera, config, scene_config);
        if (!driver.prepare()) return 4;
        double map_ms = c->caustics ? build_photon_map(driver, c) : 0.0;
        if (photon_ms) *photon_ms = map_ms;
        RenderTaskRenderer renderer(driver);
        RenderTask task;
        task.jobFingerprint = computeRenderFingerprint(config, scene_config);
        task.tile = DistributedTile{0, 0, c->width, c->height};
        for (uint32_t i = 0; i <= steps; ++i) {
            task.id = RenderTaskId{0, sample_start + i * spp, spp};
            auto t0 = std::chrono::steady_clock::now();
            RenderTaskResult result = renderer.render(task);
            auto t1 = std::chrono::steady_clock::now();
            if (!result.success) return 2;
            if (i > 0) task_ms[i - 1] = std::chrono::duration<double, std::milli>(t1 - t0).count();
            if (i == steps && rgb) std::memcpy(rgb, result.radiance.data(), sizeof(float) * 3 * result.radiance.size());
        }
        if (config.profileQueues && driver.resources_.deviceQueueCounts)
            WFCUDA_CHECK(cudaMemcpy(queue_counts, driver.resources_.deviceQueueCounts, sizeof(uint32_t) * c->max_depth,
                                    cudaMemcpyDeviceToHost));
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfcuda_render: %s\n", e.what());
        return 3;
    }
}

// The converged-image accumulator: renders `tasks` tasks of the tile
// (x, y, w, h), each `spp` samples from sample_start + i * spp on, through
// RenderTaskRenderer::render, and adds every task's FP32 sums into `sum`
// (w * h * 3 doubles) on the host.  The driver, and with c->caustics its
// photon map, is made once.
int wfcuda_render_sum(void* handle, const wf_camera* cam, const wf_render_config* c, int persistent, uint32_t x,
                      uint32_t y, uint32_t w, uint32_t h, uint32_t sample_start, uint32_t spp, uint32_t tasks,
                      double* sum) {
    try {
        CudaRefScene* r = static_cast<CudaRefScene*>(handle);
        if (!r || spp == 0 || !sum) return 1;
        Camera camera = reference_camera(cam);
        RenderConfig config = reference_config(c, persistent, false);
        SceneConfig scene_config;
        scene_config.preset = ScenePreset::Demo;
        RenderDriver driver(r->device, camera, config, scene_config);
        if (!driver.prepare()) return 4;
        if (c->caustics) build_photon_map(driver, c);
        RenderTaskRenderer renderer(driver);
        RenderTask task;
        task.jobFingerprint = computeRenderFingerprint(config, scene_config);
        task.tile = DistributedTile{x, y, w, h};
        for (uint32_t i = 0; i < tasks; ++i) {
            task.id = RenderTaskId{0, sample_start + i * spp, spp};
            RenderTaskResult result = renderer.render(task);
            if (!result.success) return 2;
            for (size_t k = 0; k < result.radiance.size(); ++k) {
                sum[3 * k] += result.radiance[k].x;
                sum[3 * k + 1] += result.radiance[k].y;
                sum[3 * k + 2] += result.radiance[k].z;
            }
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfcuda_render_sum: %s\n", e.what());
        return 3;
    }
}

}  // extern "C"
