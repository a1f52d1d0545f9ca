// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into or called by the
// product.  Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
// load the library built from this file (oracle/_ref/libwfref.so).
//
// Runs the reference's own renderer code on host threads.  The reference
// sources (src/scene/scene.cu, src/renderer/renderer.cu, photon_mapping.cu,
// src/scene/environment.cpp, src/core/rng.cu, ...) are compiled unmodified as
// host C++ by oracle/build_ref.sh; this file only converts the C-ABI scene
// description into the reference's HostScene, calls uploadScene (which, with
// the runtime stubs of ref_stubs.h, builds the device scene in host memory),
// and launches the reference kernels one host thread per CUDA thread, in the
// order RenderDriver::createWavefrontGraph records them
// (src/renderer/render_driver.cu:264-297).
#include "renderer/renderer.cuh"
#include "scene/environment.hpp"
#include "scene/scene_host.hpp"
#include "renderer/render_session.cuh"
#include "renderer/frame_guides.cuh"

#include "../include/wavefront.h"
#include "../wavefront-path-tracer_b200/csrc/bvh_build.h"
#include "ref_scene_convert.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>

thread_local WfRefDim3 blockIdx, blockDim, threadIdx, gridDim;

// Defined in the reference translation units (external linkage there).
__device__ bool isOccluded(const Ray& ray, float maximumDistance, Scene scene);
__device__ float dielectricReflectance(float cosine, float eta);
using wfref::v3;

// ------------------------------------------------------------ NXB builder
namespace {
NXB::BVH2 build_nexus(std::vector<wf::BvhBox>& boxes) {
    NXB::BVH2 bvh;
    std::vector<wf::BvhBinaryNode> nodes;
    wf::build_binary_bvh(boxes.data(), uint32_t(boxes.size()), nodes, 0);
    bvh.storage_.resize(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        const wf::BvhBinaryNode& n = nodes[i];
        bvh.storage_[i].bounds = NXB::AABB(make_float3(n.box.lo[0], n.box.lo[1], n.box.lo[2]),
                                           make_float3(n.box.hi[0], n.box.hi[1], n.box.hi[2]));
        bvh.storage_[i].leftChild = n.left;
        bvh.storage_[i].rightChild = n.right;
    }
    bvh.primCount_ = uint32_t(boxes.size());
    if (!nodes.empty()) bvh.bounds_ = bvh.storage_.back().bounds;
    return bvh;
}
}  // namespace

namespace NXB {
BVH2 BuildBVH2(const Triangle* triangles, uint32_t count, BuildConfig, BVHBuildMetrics*) {
    std::vector<wf::BvhBox> boxes(count);
    for (uint32_t i = 0; i < count; ++i) {
        const Triangle& t = triangles[i];
        boxes[i].lo[0] = std::min(std::min(t.v0.x, t.v1.x), t.v2.x);
        boxes[i].lo[1] = std::min(std::min(t.v0.y, t.v1.y), t.v2.y);
        boxes[i].lo[2] = std::min(std::min(t.v0.z, t.v1.z), t.v2.z);
        boxes[i].hi[0] = std::max(std::max(t.v0.x, t.v1.x), t.v2.x);
        boxes[i].hi[1] = std::max(std::max(t.v0.y, t.v1.y), t.v2.y);
        boxes[i].hi[2] = std::max(std::max(t.v0.z, t.v1.z), t.v2.z);
    }
    return build_nexus(boxes);
}
BVH2 BuildBVH2(const AABB* aabbs, uint32_t count, BuildConfig, BVHBuildMetrics*) {
    std::vector<wf::BvhBox> boxes(count);
    for (uint32_t i = 0; i < count; ++i) {
        boxes[i] = wf::BvhBox{{aabbs[i].bMin.x, aabbs[i].bMin.y, aabbs[i].bMin.z},
                              {aabbs[i].bMax.x, aabbs[i].bMax.y, aabbs[i].bMax.z}};
    }
    return build_nexus(boxes);
}
BVH8 BuildBVH8(const Triangle*, uint32_t, BuildConfig, BVHBuildMetrics*) {
    throw std::runtime_error("BVH8 is not provided by the NexusBVH shim");
}
}  // namespace NXB

// ------------------------------------------------------------- textures
namespace {
struct TextureRecord {
    cudaArray* array;
    cudaTextureDesc desc;
};
std::vector<TextureRecord> g_textures;  // handle = index + 1

float4 texel(const cudaArray* a, uint32_t x, uint32_t y, bool normalizedRead) {
    size_t offset = (size_t(y) * a->width + x) * a->texelBytes;
    if (a->texelBytes == 16) {
        float4 v;
        std::memcpy(&v, a->data.data() + offset, 16);
        return v;
    }
    const unsigned char* p = a->data.data() + offset;
    float s = normalizedRead ? 1.0f / 255.0f : 1.0f;
    return make_float4(p[0] * s, p[1] * s, p[2] * s, p[3] * s);
}

int address(int i, int n, cudaTextureAddressMode mode) {
    if (mode == cudaAddressModeWrap) return ((i % n) + n) % n;
    return std::clamp(i, 0, n - 1);
}
}  // namespace

float4 wfref_texture_fetch(cudaTextureObject_t object, float u, float v) {
    const TextureRecord& r = g_textures.at(size_t(object) - 1);
    const cudaArray* a = r.array;
    float tx = u * a->width - .5f, ty = v * a->height - .5f;
    int x = int(floorf(tx)), y = int(floorf(ty));
    float fx = tx - x, fy = ty - y;
    float4 result{};
    bool normalizedRead = r.desc.readMode == cudaReadModeNormalizedFloat;
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            int xx = address(x + i, int(a->width), r.desc.addressMode[0]);
            int yy = address(y + j, int(a->height), r.desc.addressMode[1]);
            float4 p = texel(a, uint32_t(xx), uint32_t(yy), normalizedRead);
            float w = (i ? fx : 1 - fx) * (j ? fy : 1 - fy);
            result.x += w * p.x;
            result.y += w * p.y;
            result.z += w * p.z;
            result.w += w * p.w;
        }
    return result;
}

cudaError_t wfref_cudaMallocArray(cudaArray_t* array, const cudaChannelFormatDesc* desc, size_t width,
                                  size_t height, unsigned int) {
    cudaArray* a = new cudaArray;
    a->width = uint32_t(width);
    a->height = uint32_t(height);
    a->desc = *desc;
    a->texelBytes = size_t(desc->x + desc->y + desc->z + desc->w) / 8;
    a->data.resize(a->texelBytes * width * height);
    *array = a;
    return cudaSuccess;
}
cudaError_t wfref_cudaMemcpy2DToArray(cudaArray_t array, size_t, size_t, const void* src, size_t spitch,
                                      size_t width, size_t height, cudaMemcpyKind) {
    for (size_t row = 0; row < height; ++row)
        std::memcpy(array->data.data() + row * width, static_cast<const char*>(src) + row * spitch, width);
    return cudaSuccess;
}
cudaError_t wfref_cudaFreeArray(cudaArray_t array) {
    delete array;
    return cudaSuccess;
}
cudaError_t wfref_cudaCreateTextureObject(cudaTextureObject_t* object, const cudaResourceDesc* resource,
                                          const cudaTextureDesc* texture, const cudaResourceViewDesc*) {
    g_textures.push_back(TextureRecord{resource->res.array.array, *texture});
    *object = cudaTextureObject_t(g_textures.size());
    return cudaSuccess;
}
cudaError_t wfref_cudaDestroyTextureObject(cudaTextureObject_t) { return cudaSuccess; }

// --------------------------------------------------------- host "launch"
namespace {
template <typename F>
void parallel_for(uint32_t count, int threads, F&& body) {
    if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
    threads = int(std::min<uint32_t>(uint32_t(threads), std::max(1u, count / 64 + 1)));
    std::atomic<uint32_t> next{0};
    auto worker = [&] {
        blockDim.x = 1;
        threadIdx.x = 0;
        gridDim.x = count;
        for (;;) {
            uint32_t begin = next.fetch_add(64);
            if (begin >= count) break;
            uint32_t end = std::min(count, begin + 64);
            for (uint32_t i = begin; i < end; ++i) {
                blockIdx.x = i;
                body(i);
            }
        }
    };
    if (threads == 1) { worker(); return; }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
}

}  // namespace
struct RefPhotonMap;
namespace {
struct RefScene {
    DeviceScene device;
    uint32_t original_material_count = 0;
    bool probe = false;
    std::shared_ptr<RefPhotonMap> photons;  // cached map (built once, like RenderDriver::prepare)
    std::string photon_key;
};
}  // namespace

// ------------------------------------------------------------- C API
extern "C" {

// probe != 0 builds the hit-identity probe copy: light registration off,
// triangle lightIndex = identity code, instance lightOffset = index << 24,
// material overrides baked into per-instance mesh copies, one private
// material per sphere.
void* wfref_scene_create(const wf_scene_desc* d, const wf_environment* env, int probe) {
    try {
        HostScene h;
        auto r = std::make_unique<RefScene>();
        r->probe = probe != 0;
        wfref::host_scene_from_desc(d, probe != 0, h);
        r->original_material_count = d->material_count;
        r->device = uploadScene(h);
        r->device.scene.ignoreDirectLightOcclusion = d->ignore_direct_light_occlusion != 0;
        wfref::apply_normal_map_settings(r->device.scene, d);
        if (probe) {
            for (uint32_t i = 0; i < r->device.scene.instanceCount; ++i)
                r->device.instances[i].lightOffset = i << 24;
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
        return r.release();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfref_scene_create: %s\n", e.what());
        return nullptr;
    }
}

HostScene* wfref_host_scene_get(void* host);  // ref_assets.cpp

// A renderable reference scene from a HostScene that the reference's own
// loaders and preset assembly built (ref_assets.cpp).  Its BVH2s go through
// the same NexusBVH builder as scenes from a description.
void* wfref_scene_from_host(void* host, int disable_normal_maps, float normal_map_minimum_cosine) {
    try {
        HostScene h = *wfref_host_scene_get(host);
        h.acceleration = ObjAccelerationPolicy::NexusBvh2;
        auto r = std::make_unique<RefScene>();
        r->original_material_count = uint32_t(h.materials.size());
        r->device = uploadScene(h);
        r->device.scene.useNormalMaps = disable_normal_maps == 0;
        r->device.scene.normalMapMinimumCosine = normal_map_minimum_cosine;
        return r.release();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfref_scene_from_host: %s\n", e.what());
        return nullptr;
    }
}

void wfref_scene_destroy(void* handle) {
    RefScene* r = static_cast<RefScene*>(handle);
    if (!r) return;
    destroyDeviceScene(r->device);
    delete r;
}

uint32_t wfref_scene_light_count(void* handle) {
    return static_cast<RefScene*>(handle)->device.scene.lightCount;
}

// 16 floats per light: v0 v1 v2 normal (12), area, material, selectionPdf,
// alias probability; plus alias index in `alias`.
void wfref_scene_lights(void* handle, float* lights, uint32_t* alias) {
    const Scene& s = static_cast<RefScene*>(handle)->device.scene;
    for (uint32_t i = 0; i < s.lightCount; ++i) {
        const TriangleLight& l = s.lights[i];
        float* o = lights + 16 * size_t(i);
        const Vec3 v[4] = {l.v0, l.v1, l.v2, l.normal};
        for (int k = 0; k < 4; ++k) { o[3 * k] = v[k].x; o[3 * k + 1] = v[k].y; o[3 * k + 2] = v[k].z; }
        o[12] = l.area;
        std::memcpy(&o[13], &l.material, 4);
        o[14] = l.selectionPdf;
        o[15] = s.lightAlias[i].probability;
        alias[i] = s.lightAlias[i].alias;
    }
}

// Environment distribution built by the reference (environment.cpp:10-64).
int wfref_environment_distribution(const float* rgba, uint32_t width, uint32_t height, float* probabilities,
                                   float* alias_probability, uint32_t* alias) {
    try {
        HostEnvironment map;
        map.width = width;
        map.height = height;
        map.pixels.resize(size_t(width) * height);
        for (size_t i = 0; i < map.pixels.size(); ++i)
            map.pixels[i] = make_float4(rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]);
        buildEnvironmentDistribution(map);
        for (size_t i = 0; i < map.pixels.size(); ++i) {
            probabilities[i] = map.probabilities[i];
            alias_probability[i] = map.alias[i].probability;
            alias[i] = map.alias[i].alias;
        }
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// traceRay for a batch of rays.  Probe scenes also decode the identity.
void wfref_trace(void* handle, const wf_ray* rays, uint32_t count, wf_hit* hits, int threads) {
    RefScene* r = static_cast<RefScene*>(handle);
    Scene scene = r->device.scene;
    parallel_for(count, threads, [&](uint32_t i) {
        Ray ray(v3(rays[i].origin), v3(rays[i].direction));
        TraceResult res = traceRayExternal(ray, scene);
        wf_hit& o = hits[i];
        std::memset(&o, 0, sizeof(o));
        o.instance = 0xffffffffu;
        o.primitive = 0xffffffffu;
        if (!res.didHit) {
            o.material = WF_NO_MATERIAL;
            o.light_index = 0xffffffffu;
            o.kind = WF_HIT_NONE;
            o.t = 1e30f;
            return;
        }
        const Hit& h = res.hit;
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
    });
}

void wfref_occluded(void* handle, const wf_ray* rays, const float* max_distance, uint32_t count,
                    uint8_t* occluded, int threads) {
    Scene scene = static_cast<RefScene*>(handle)->device.scene;
    parallel_for(count, threads, [&](uint32_t i) {
        Ray ray(v3(rays[i].origin), v3(rays[i].direction));
        occluded[i] = isOccluded(ray, max_distance[i], scene) ? 1 : 0;
    });
}

// Photon map of the reference (emitPhotons/tracePhotons/buildPhotonGrid,
// photon_mapping.cu:4-89, driven as render_driver.cu:180-234 does).
struct RefPhotonMap {
    std::vector<Photon> photons;
    std::vector<uint32_t> heads, next;
    PhotonGrid grid{};
    uint32_t stored = 0;
};

static RefPhotonMap* build_photons(Scene scene, const wf_render_config* c, int threads) {
    auto map = std::make_unique<RefPhotonMap>();
    uint32_t n = c->photon_count;
    map->photons.resize(n);
    PhotonQueue queue{map->photons.data(), nullptr, n};
    uint32_t counts[3] = {0, 0, 0};
    RngStrategy strategy = RngStrategy(c->rng);
    parallel_for(n, threads, [&](uint32_t) {
        emitPhotons(queue, scene, n, c->photon_seed, strategy, c->spectral != 0);
    });
    parallel_for(n, threads, [&](uint32_t) { tracePhotons(queue, scene, n, c->photon_max_depth, counts); });
    map->grid.photons = map->photons.data();
    map->grid.resolution = c->photon_grid_resolution;
    map->grid.minimum = v3(c->photon_grid_min);
    map->grid.maximum = v3(c->photon_grid_max);
    bool derive = c->photon_grid_min[0] == c->photon_grid_max[0] && c->photon_grid_min[1] == c->photon_grid_max[1] &&
                  c->photon_grid_min[2] == c->photon_grid_max[2];
    if (derive) {
        // The build's grid bounds are the bounding box of the stored photons
        // (the reference hard-codes Cornell bounds, render_driver.cu:211-213);
        // degenerate axes get unit extent.
        Vec3 lo(INFINITY, INFINITY, INFINITY), hi(-INFINITY, -INFINITY, -INFINITY);
        bool any = false;
        for (const Photon& p : map->photons) {
            if (!p.valid) continue;
            any = true;
            lo = Vec3(fminf(lo.x, p.position.x), fminf(lo.y, p.position.y), fminf(lo.z, p.position.z));
            hi = Vec3(fmaxf(hi.x, p.position.x), fmaxf(hi.y, p.position.y), fmaxf(hi.z, p.position.z));
        }
        if (!any) {
            lo = Vec3(-1, -1, -1);
            hi = Vec3(1, 1, 1);
        }
        if (!(hi.x > lo.x)) hi.x = lo.x + 1.0f;
        if (!(hi.y > lo.y)) hi.y = lo.y + 1.0f;
        if (!(hi.z > lo.z)) hi.z = lo.z + 1.0f;
        map->grid.minimum = lo;
        map->grid.maximum = hi;
    }
    size_t cells = size_t(c->photon_grid_resolution) * c->photon_grid_resolution * c->photon_grid_resolution;
    map->heads.assign(cells, 0xffffffffu);
    map->next.assign(n, 0xffffffffu);
    map->grid.heads = map->heads.data();
    map->grid.next = map->next.data();
    // Serial insertion keeps every cell list in increasing photon order, so the
    // gather is deterministic (the device builds the same lists in atomic order).
    blockDim.x = 1; threadIdx.x = 0;
    for (uint32_t i = 0; i < n; ++i) {
        blockIdx.x = i;
        buildPhotonGrid(queue, map->grid, n);
    }
    for (const Photon& p : map->photons) map->stored += p.valid ? 1 : 0;
    return map.release();
}

// Photon records: 8 floats (position, direction, flux sum, valid) + flux rgb
// in `flux` (3 floats) per emitted photon.
int wfref_photons(void* handle, const wf_render_config* c, float* records, float* flux, uint32_t* stored,
                  int threads) {
    Scene scene = static_cast<RefScene*>(handle)->device.scene;
    std::unique_ptr<RefPhotonMap> map(build_photons(scene, c, threads));
    for (uint32_t i = 0; i < c->photon_count; ++i) {
        const Photon& p = map->photons[i];
        float* o = records + 8 * size_t(i);
        o[0] = p.position.x; o[1] = p.position.y; o[2] = p.position.z;
        o[3] = p.direction.x; o[4] = p.direction.y; o[5] = p.direction.z;
        o[6] = p.flux.x + p.flux.y + p.flux.z;
        o[7] = p.valid ? 1.0f : 0.0f;
        if (flux) { flux[3 * i] = p.flux.x; flux[3 * i + 1] = p.flux.y; flux[3 * i + 2] = p.flux.z; }
    }
    *stored = map->stored;
    return 0;
}

// Renders absolute samples [sample_start, sample_start + sample_count) of a
// tile with the reference's captured-graph kernel chain (or, persistent != 0,
// its cooperative persistent kernel on a single host worker).  fb32 receives
// the FP32 framebuffer sums exactly as the reference accumulates them;
// fb64 (nullable) the per-sample radiance summed in FP64.  queue_counts
// (nullable) receives max_depth counts per sample (sample-major).
// generateFrameGuides (device_frame_guides.cuh:6-41) as host code, one host
// worker per CUDA thread, over the tile (x, y, w, h) of a width x height
// image; out receives w*h FrameGuide records.  prev may be NULL.
int wfref_frame_guides(void* handle, const wf_camera* cam, const wf_camera* prev, uint32_t width, uint32_t height,
                       uint32_t x, uint32_t y, uint32_t w, uint32_t h, wf_frame_guide* out, int threads) {
    static_assert(sizeof(FrameGuide) == sizeof(wf_frame_guide), "FrameGuide layout");
    RefScene* r = static_cast<RefScene*>(handle);
    if (!r || !cam || !out) return 1;
    auto camera = [](const wf_camera* c) {
        Camera k;
        k.position = v3(c->position);
        k.forward = v3(c->forward);
        k.right = v3(c->right);
        k.up = v3(c->up);
        k.verticalFov = c->vertical_fov;
        k.aspectRatio = c->aspect_ratio;
        return k;
    };
    Scene scene = r->device.scene;
    Camera now = camera(cam);
    Camera before = prev ? camera(prev) : now;
    RenderTile tile{x, y, w, h, 1};
    std::vector<FrameGuide> guides(size_t(w) * h);
    parallel_for(w * h, threads, [&](uint32_t) {
        generateFrameGuides(guides.data(), scene, now, before, prev != nullptr, width, height, tile);
    });
    std::memcpy(out, guides.data(), sizeof(FrameGuide) * guides.size());
    return 0;
}

int wfref_render(void* handle, const wf_camera* cam, const wf_render_config* c, uint32_t x0, uint32_t y0,
                 uint32_t tw, uint32_t th, uint32_t sample_start, uint32_t sample_count, float* fb32,
                 double* fb64, uint32_t* queue_counts, int threads, int persistent) {
    try {
        RefScene* r = static_cast<RefScene*>(handle);
        Scene scene = r->device.scene;
        Camera camera;
        camera.position = v3(cam->position);
        camera.forward = v3(cam->forward);
        camera.right = v3(cam->right);
        camera.up = v3(cam->up);
        camera.verticalFov = cam->vertical_fov;
        camera.aspectRatio = cam->aspect_ratio;
        uint32_t width = c->width, height = c->height;
        uint32_t capacity = tw * th;
        std::vector<PathState> paths(capacity);
        std::vector<RayWorkItem> raysA(capacity), raysB(capacity);
        std::vector<IntersectionResult> results(capacity);
        uint32_t countA = 0, countB = 0;
        std::vector<Vec3> framebuffer(size_t(width) * height);
        std::vector<Vec3> sampleBuffer(size_t(width) * height);
        RenderTile tile{x0, y0, tw, th, 1};
        uint32_t sampleIndex = 0;
        RngStrategy strategy = RngStrategy(c->rng);
        bool intersectionDebug = c->debug == WF_DEBUG_INTERSECTION;
        bool normalDebug = c->debug == WF_DEBUG_SHADING_NORMAL;
        PhotonGrid shadingGrid{};
        if (c->caustics && c->photon_count) {
            char key[256];
            std::snprintf(key, sizeof(key), "%u/%u/%u/%u/%u/%u/%a/%a/%a/%a/%a/%a", c->photon_count, c->photon_seed,
                          c->photon_max_depth, c->photon_grid_resolution, c->rng, c->spectral,
                          c->photon_grid_min[0], c->photon_grid_min[1], c->photon_grid_min[2],
                          c->photon_grid_max[0], c->photon_grid_max[1], c->photon_grid_max[2]);
            if (!r->photons || r->photon_key != key) {
                r->photons.reset(build_photons(scene, c, threads));
                r->photon_key = key;
            }
            shadingGrid = r->photons->grid;
            if (!c->caustic_gather) shadingGrid.heads = nullptr;
        }
        std::vector<uint32_t> counts(c->max_depth);
        for (uint32_t s = 0; s < sample_count; ++s) {
            sampleIndex = sample_start + s;
            std::fill(sampleBuffer.begin(), sampleBuffer.end(), Vec3());
            std::fill(counts.begin(), counts.end(), 0u);
            RayQueue first{raysA.data(), &countA, capacity};
            RayQueue second{raysB.data(), &countB, capacity};
            if (persistent) {
                blockIdx.x = 0; blockDim.x = 1; threadIdx.x = 0; gridDim.x = 1;
                persistentWavefrontTrace(first, second, paths.data(), counts.data(), camera, width, height,
                                         &sampleIndex, &tile, strategy, scene, c->max_depth,
                                         c->rr_start_depth, intersectionDebug, normalDebug,
                                         sampleBuffer.data(), shadingGrid, c->gather_radius,
                                         c->indirect_clamp);
            } else {
                countA = 0;
                parallel_for(capacity, threads, [&](uint32_t) {
                    generatePrimaryRays(first, paths.data(), camera, width, height, &sampleIndex, &tile,
                                        strategy, c->indirect_clamp);
                });
                RayQueue current = first, next = second;
                for (uint32_t bounce = 0; bounce < c->max_depth; ++bounce) {
                    uint32_t n = *current.count;
                    counts[bounce] = n;
                    *next.count = 0;
                    parallel_for(n, threads, [&](uint32_t) {
                        intersectScene(current, results.data(), scene);
                    });
                    parallel_for(n, threads, [&](uint32_t) {
                        shadePaths(current, results.data(), next, paths.data(), scene, c->max_depth,
                                   c->rr_start_depth, intersectionDebug, normalDebug, sampleBuffer.data(),
                                   shadingGrid, c->gather_radius);
                    });
                    std::swap(current, next);
                }
            }
            for (uint32_t y = y0; y < y0 + th; ++y)
                for (uint32_t x = x0; x < x0 + tw; ++x) {
                    size_t p = size_t(y) * width + x;
                    framebuffer[p] += sampleBuffer[p];
                    size_t o = (size_t(y - y0) * tw + (x - x0)) * 3;
                    if (fb64) {
                        fb64[o] += sampleBuffer[p].x;
                        fb64[o + 1] += sampleBuffer[p].y;
                        fb64[o + 2] += sampleBuffer[p].z;
                    }
                }
            if (queue_counts)
                std::memcpy(queue_counts + size_t(s) * c->max_depth, counts.data(), 4 * size_t(c->max_depth));
        }
        for (uint32_t y = y0; y < y0 + th; ++y)
            for (uint32_t x = x0; x < x0 + tw; ++x) {
                size_t p = size_t(y) * width + x;
                size_t o = (size_t(y - y0) * tw + (x - x0)) * 3;
                fb32[o] = framebuffer[p].x;
                fb32[o + 1] = framebuffer[p].y;
                fb32[o + 2] = framebuffer[p].z;
            }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfref_render: %s\n", e.what());
        return 1;
    }
}

// The ray queues of one sample of a tile through the reference's captured
// chain (generatePrimaryRays, then intersectScene + shadePaths per bounce,
// renderer.cu:10-42, device_path_shading.cuh:6-173): the camera rays
// (bounce 0) and the continuation rays each bounce appends, for `bounces`
// queues.  rays receives them back to back (capacity ray_capacity), in queue
// order; counts[b] the size of queue b.  Caustics are not gathered (the
// queues do not depend on them).  Returns the number of rays written, or
// ~0u on an error or an overflow of ray_capacity.
uint32_t wfref_path_rays(void* handle, const wf_camera* cam, const wf_render_config* c, uint32_t x0, uint32_t y0,
                         uint32_t tw, uint32_t th, uint32_t sample, uint32_t bounces, wf_ray* rays,
                         uint32_t ray_capacity, uint32_t* counts, int threads) {
    try {
        RefScene* r = static_cast<RefScene*>(handle);
        Scene scene = r->device.scene;
        Camera camera;
        camera.position = v3(cam->position);
        camera.forward = v3(cam->forward);
        camera.right = v3(cam->right);
        camera.up = v3(cam->up);
        camera.verticalFov = cam->vertical_fov;
        camera.aspectRatio = cam->aspect_ratio;
        uint32_t width = c->width, height = c->height;
        uint32_t capacity = tw * th;
        std::vector<PathState> paths(capacity);
        std::vector<RayWorkItem> raysA(capacity), raysB(capacity);
        std::vector<IntersectionResult> results(capacity);
        std::vector<Vec3> sampleBuffer(size_t(width) * height);
        uint32_t countA = 0, countB = 0;
        RenderTile tile{x0, y0, tw, th, 1};
        uint32_t sampleIndex = sample;
        RngStrategy strategy = RngStrategy(c->rng);
        RayQueue current{raysA.data(), &countA, capacity};
        RayQueue next{raysB.data(), &countB, capacity};
        parallel_for(capacity, threads, [&](uint32_t) {
            generatePrimaryRays(current, paths.data(), camera, width, height, &sampleIndex, &tile, strategy,
                                c->indirect_clamp);
        });
        uint32_t written = 0;
        for (uint32_t b = 0; b < bounces; ++b) {
            uint32_t n = *current.count;
            counts[b] = n;
            if (written + n > ray_capacity) return ~0u;
            for (uint32_t i = 0; i < n; ++i) {
                const Ray& ray = current.items[i].ray;
                wf_ray& out = rays[written + i];
                out.origin[0] = ray.origin.x; out.origin[1] = ray.origin.y; out.origin[2] = ray.origin.z;
                out.direction[0] = ray.direction.x; out.direction[1] = ray.direction.y;
                out.direction[2] = ray.direction.z;
            }
            written += n;
            if (b + 1 == bounces) break;
            *next.count = 0;
            parallel_for(n, threads, [&](uint32_t) { intersectScene(current, results.data(), scene); });
            parallel_for(n, threads, [&](uint32_t) {
                shadePaths(current, results.data(), next, paths.data(), scene, c->max_depth, c->rr_start_depth,
                           false, false, sampleBuffer.data(), PhotonGrid{}, c->gather_radius);
            });
            std::swap(current, next);
        }
        return written;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfref_path_rays: %s\n", e.what());
        return ~0u;
    }
}

float wfref_dielectric_reflectance(float cosine, float eta) { return dielectricReflectance(cosine, eta); }

// The reference's checkpoint reader/writer (render_checkpoint.cpp), for
// byte-compatibility tests of the product's checkpoint files.
int wfref_checkpoint_roundtrip_read(const char* path, uint32_t width, uint32_t height, uint64_t fingerprint,
                                    float* rgb, uint32_t* sample_index) {
    RenderSession session = createRenderSession(width, height);
    *sample_index = loadRenderSessionCheckpoint(session, path, fingerprint);
    std::memcpy(rgb, session.deviceFramebuffer, sizeof(Vec3) * size_t(width) * height);
    destroyRenderSession(session);
    return 0;
}

int wfref_checkpoint_write(const char* path, uint32_t width, uint32_t height, uint64_t fingerprint,
                           const float* rgb, uint32_t sample_index) {
    RenderSession session = createRenderSession(width, height);
    std::memcpy(session.deviceFramebuffer, rgb, sizeof(Vec3) * size_t(width) * height);
    AsyncCheckpointWriter* writer = createAsyncCheckpointWriter(width, height, path, 1, fingerprint);
    bool ok = enqueueRenderSessionCheckpoint(*writer, session, sample_index, nullptr);
    finishAsyncCheckpointWriter(*writer);
    destroyAsyncCheckpointWriter(writer);
    destroyRenderSession(session);
    return ok ? 0 : 1;
}

}  // extern "C"

// The runtime's channel-descriptor helper, used by cudaCreateChannelDesc<T>()
// in the reference's texture uploads (scene.cu:49,317).
extern "C" cudaChannelFormatDesc cudaCreateChannelDesc(int x, int y, int z, int w, cudaChannelFormatKind f) {
    cudaChannelFormatDesc d;
    d.x = x; d.y = y; d.z = z; d.w = w; d.f = f;
    return d;
}

extern "C" {
// Draws n floats from the reference RNG (makeRngState + randomFloat,
// include/core/rng.cuh:15-29, src/core/rng.cu:29-42) keyed by pixelRngKey.
void wfref_rng(uint32_t pixel, uint32_t sample, uint32_t strategy, uint32_t n, float* out, uint64_t* state) {
    RngState s = makeRngState(pixelRngKey(pixel, sample, RngStrategy(strategy)), RngStrategy(strategy));
    if (state) *state = s.state;
    for (uint32_t i = 0; i < n; ++i) out[i] = randomFloat(s);
}

// The elementary functions as this build of the reference evaluates them
// (C library, or wf_math.h in libwfref_det.so).  kind: 0 sinf 1 cosf 2 tanf
// 3 atan2f 4 logf 5 expf 6 powf 7 sin 8 cos.
void wfref_math(int kind, const float* x, const float* y, uint32_t n, double* out) {
    for (uint32_t i = 0; i < n; ++i) {
        switch (kind) {
        case 0: out[i] = sinf(x[i]); break;
        case 1: out[i] = cosf(x[i]); break;
        case 2: out[i] = tanf(x[i]); break;
        case 3: out[i] = atan2f(x[i], y[i]); break;
        case 4: out[i] = logf(x[i]); break;
        case 5: out[i] = expf(x[i]); break;
        case 6: out[i] = powf(x[i], y[i]); break;
        case 7: out[i] = sin(double(x[i])); break;
        default: out[i] = cos(double(x[i])); break;
        }
    }
}
}
