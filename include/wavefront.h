/*
 * wavefront.h -- C ABI of the B200 wavefront path tracer.
 *
 * Every entry point takes plain pointers and sizes, returns a wf_status and
 * never exits the process.  Objects are not thread-safe: use one renderer per
 * host thread.  All device work of a renderer runs on the stream it was
 * created with.
 *
 * Each declaration cites the reference interface it replaces
 * (Gh05ts/Wavefront-Path-Tracer, paths relative to that project).
 */
#ifndef WAVEFRONT_H
#define WAVEFRONT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef int32_t wf_status;
enum {
    WF_OK = 0,
    WF_ERR_INVALID_ARG = 1,
    WF_ERR_OOM = 2,
    WF_ERR_CUDA = 3,
    WF_ERR_TIMEOUT = 4,
    WF_ERR_FINGERPRINT = 5,
    WF_ERR_CAPACITY = 6,
    WF_ERR_IO = 7,
    WF_ERR_FORMAT = 8,
    WF_ERR_UNSUPPORTED = 9,
    WF_ERR_STATE = 10
};

/* Thread-local text of the last error reported by this library. */
const char* wf_last_error(void);
/* Library version string ("wavefront-b200 <major>.<minor>"). */
const char* wf_version(void);

/* Testing hook (no counterpart in the reference, which exits on a failed
 * cudaMalloc): the library's next `after` device allocations succeed and the
 * one after them fails with cudaErrorMemoryAllocation, once; the entry point
 * that made it frees what it had allocated and returns WF_ERR_OOM.  A
 * negative value disarms the hook.  Process-wide. */
void wf_test_fail_allocation(int64_t after);

/* ------------------------------------------------------------------ scene */
/* MaterialType, include/scene/material.cuh:22-28 */
enum { WF_MAT_DIFFUSE = 0, WF_MAT_METAL = 1, WF_MAT_DIELECTRIC = 2,
       WF_MAT_EMISSIVE = 3, WF_MAT_SPECGLOSS = 4 };
/* AccelerationMode, include/scene/scene.cuh:21 (Bvh = 0, Direct = 1) */
enum { WF_ACCEL_BVH = 0, WF_ACCEL_DIRECT = 1 };
/* PunctualLightType, include/scene/punctual_light.cuh:6 */
enum { WF_LIGHT_POINT = 0, WF_LIGHT_SPOT = 1, WF_LIGHT_DIRECTIONAL = 2 };
enum { WF_NO_MATERIAL = 0xffffffffu };

/* Material, include/scene/material.cuh:30-70 (texture bindings are not
 * carried: every material is untextured, so texture lookups return the
 * factors exactly as device_traversal.cuh:351-356 does without a texture). */
typedef struct wf_material {
    uint32_t type;
    float albedo[3];
    float emission[3];
    float roughness;
    float ior;
    float dispersion;
    float metallic;
    float attenuation_color[3];
    float attenuation_distance;
    float volume_density;
    float opacity;
    float alpha_cutoff;
    uint32_t alpha_masked;
    uint32_t specgloss_workflow;
    uint32_t gltf_pbr;
    float specular[3];
    float glossiness;
    float specular_weight;
    float specular_color[3];
    float clearcoat;
    float clearcoat_roughness;
} wf_material;

/* Fills the reference's default member values (material.cuh:30-70) with
 * roughness 0 and ior 1 as makeMaterial sets them (src/scene/scene_host.cpp:44-52). */
void wf_material_default(wf_material* material, uint32_t type);

/* Triangle, include/scene/geometry.cuh:13-45: positions, optional vertex
 * normals and material.  Texture coordinates and tangent frames, which only
 * textured materials read, come in an optional parallel array
 * (wf_triangle_attributes). */
typedef struct wf_triangle {
    float v0[3], v1[3], v2[3];
    float n0[3], n1[3], n2[3];
    uint32_t material;
    uint32_t has_vertex_normals;
} wf_triangle;

/* SceneSphere, include/scene/scene_host.hpp:8-14 */
typedef struct wf_sphere {
    float center[3];
    float radius;
    uint32_t material;
    uint32_t accel; /* WF_ACCEL_BVH: TLAS leaf; WF_ACCEL_DIRECT: tested directly */
} wf_sphere;

/* MeshAsset, include/scene/scene.cuh:117-119 */
/* The texture coordinates and tangent frames of a Triangle,
 * include/scene/geometry.cuh:22-41 (uv0-uv2, uv1_0-uv1_2, tangent,
 * bitangent, tangent1, bitangent1, vertexTangent0-2, vertexTangentSign0-2,
 * hasVertexTangents, hasTexcoords, hasTexcoords1; geometry.cuh:22-48).
 * Without has_texcoords (has_texcoords1) a set reads as (0, 0). */
typedef struct wf_triangle_attributes {
    float uv[3][2];
    float uv1[3][2];
    float tangent[3], bitangent[3], tangent1[3], bitangent1[3];
    float vertex_tangent[3][3];
    float vertex_tangent_sign[3];
    uint32_t has_vertex_tangents;
    uint32_t has_texcoords;
    uint32_t has_texcoords1;
} wf_triangle_attributes;

typedef struct wf_mesh {
    const wf_triangle* triangles;
    uint32_t triangle_count;
    const wf_triangle_attributes* attributes; /* NULL, or triangle_count records */
} wf_mesh;

#define WF_NO_TEXTURE 0xffffffffu

/* ObjTexture, include/scene/obj_loader.hpp:9-13: RGBA8 texels, row-major
 * from the first stored row; sampled with wrapping and bilinear filtering
 * at (u, 1 - v) (src/scene/scene.cu:44-80, device_traversal.cuh:341-347). */
typedef struct wf_texture {
    uint32_t width, height;
    const uint8_t* rgba;
} wf_texture;

/* TextureBinding, include/scene/material.cuh:14-21 (KHR_texture_transform). */
typedef struct wf_texture_binding {
    uint32_t texture;  /* WF_NO_TEXTURE, or an index into wf_scene_desc::textures */
    uint32_t texcoord; /* 0 or 1 */
    float offset[2];
    float scale[2];
    float rotation;
    uint32_t has_transform;
} wf_texture_binding;

/* The texture bindings of a Material, include/scene/material.cuh:42-69, and
 * its normal-map scales. */
typedef struct wf_material_textures {
    float normal_scale;           /* Material::normalScale (1) */
    float clearcoat_normal_scale; /* Material::clearcoatNormalScale (1) */
    wf_texture_binding albedo, metallic_roughness, emissive, normal, thickness, specular_glossiness,
        specular_weight, specular_color, clearcoat, clearcoat_roughness, clearcoat_normal;
} wf_material_textures;

/* SceneInstance + InstanceTransform, include/scene/scene.cuh:27-35,121-126.
 * local_to_world[i] / world_to_local[i] are the reference's X, Y, Z basis
 * vectors (localToWorldX = local_to_world[0], ...). */
typedef struct wf_instance {
    uint32_t mesh;
    uint32_t material_override; /* WF_NO_MATERIAL = none */
    uint32_t accel;
    float local_to_world[3][3];
    float world_to_local[3][3];
    float translation[3];
} wf_instance;

/* PunctualLight, include/scene/punctual_light.cuh:8-16 */
typedef struct wf_punctual_light {
    uint32_t type;
    float position[3];
    float direction[3];
    float intensity[3];
    float range;
    float inner_cone_cos;
    float outer_cone_cos;
} wf_punctual_light;

/* HostEnvironment pixels (include/scene/environment.hpp:6-11): width*height
 * RGBA float texels, row 0 = top (+Y). */
typedef struct wf_environment {
    uint32_t width;
    uint32_t height;
    const float* rgba;
    float intensity;
    float rotation_degrees;
} wf_environment;

/* HostScene, include/scene/scene_host.hpp:19-33 */
typedef struct wf_scene_desc {
    const wf_sphere* spheres;
    uint32_t sphere_count;
    const wf_triangle* triangles;        /* HostScene::triangles (own BVH2) */
    uint32_t triangle_count;
    const wf_triangle* static_triangles; /* HostScene::staticTriangles (linear) */
    uint32_t static_triangle_count;
    const wf_mesh* meshes;
    uint32_t mesh_count;
    const wf_instance* instances;
    uint32_t instance_count;
    const wf_material* materials;
    uint32_t material_count;
    const wf_punctual_light* punctual_lights;
    uint32_t punctual_light_count;
    uint32_t black_background;
    uint32_t ignore_direct_light_occlusion;
    /* 1 = register emissive mesh and static triangles as NEE lights in the
     * order the reference's scene assembly does (addMeshTriangleLights then
     * addStaticTriangleLights, src/scene/scene_host.cpp:60-106). */
    uint32_t register_triangle_lights;
    uint32_t build_threads; /* 0 = all host threads */
    /* WF_BVH_HOST_SAH (0, default): binned-SAH BVH2s built on the host.
     * WF_BVH_GPU_PLOC: BVH2s over >= 4096 primitives built on the GPU by
     * PLOC and treelet restructuring, with the levels above 16-leaf
     * subtrees rebuilt by the host builder (the role of the reference's
     * NexusBVH builder, scene.cu:148-149, 227-228, 262-264); smaller ones,
     * and any build that fails or exceeds the 60-level depth bound, use the
     * host builder.  No counterpart field in the reference. */
    uint32_t bvh_builder;
    uint32_t reserved;
    /* Textured materials (all optional): RGBA8 textures, one
     * wf_material_textures per material, and the attributes of `triangles`
     * and `static_triangles` (those of mesh triangles are in wf_mesh).
     * Scene::useNormalMaps and normalMapMinimumCosine
     * (include/scene/scene.cuh:159-160): normal maps apply unless
     * disable_normal_maps is set. */
    const wf_texture* textures;
    uint32_t texture_count;
    uint32_t disable_normal_maps;
    const wf_material_textures* material_textures;
    const wf_triangle_attributes* triangle_attributes;
    const wf_triangle_attributes* static_triangle_attributes;
    float normal_map_minimum_cosine;
    uint32_t reserved2;
} wf_scene_desc;

enum { WF_BVH_HOST_SAH = 0, WF_BVH_GPU_PLOC = 1 };

typedef struct wf_scene wf_scene;

/* Host-side acceleration/light build + device upload.
 * Replaces DeviceScene uploadScene(const HostScene&), src/scene/scene.cu:336-389. */
wf_status wf_scene_create(const wf_scene_desc* desc, wf_scene** out);
/* Replaces uploadEnvironmentMap(DeviceScene&, const HostEnvironment&, float, float),
 * src/scene/scene.cu:308-334, including buildEnvironmentDistribution
 * (src/scene/environment.cpp:10-64).  env == NULL clears the map
 * (clearEnvironmentMap, scene.cu:298-306). */
wf_status wf_scene_set_environment(wf_scene* scene, const wf_environment* env);
/* Sets the RGB albedo of `count` materials (host arrays: material indices,
 * and 3 floats each) in the device scene, in place.  Waits until the device
 * is idle first; every renderer made from the scene renders with the new
 * albedos from its next call on.  Photon maps that renderers built at
 * creation are not retraced.  For inverse rendering with
 * wf_render_albedo_gradient; no counterpart in the reference. */
wf_status wf_scene_set_albedos(wf_scene* scene, const uint32_t* materials, const float* rgb, uint32_t count);
/* Replaces destroyDeviceScene, src/scene/scene.cu:391-420. */
wf_status wf_scene_destroy(wf_scene* scene);

typedef struct wf_scene_info {
    uint32_t light_count;
    uint32_t tlas_leaf_count;
    uint32_t blas_count;
    uint32_t material_count;
    uint64_t device_bytes;
    double build_seconds;
    uint32_t gpu_bvh_builds;  /* BVH2s the GPU builder produced */
    float bvh_build_ms;       /* wall time of all BVH2 builds of the scene */
} wf_scene_info;
wf_status wf_scene_get_info(const wf_scene* scene, wf_scene_info* info);

/* Builds one binary BVH2 over `count` boxes (6 floats each: lo xyz, hi xyz)
 * with WF_BVH_HOST_SAH or WF_BVH_GPU_PLOC (on the current device) and writes
 * its 2*count-1 nodes, 8 words each: box (6 floats), left, right.  A leaf has
 * left = 0xffffffff and right = its box index; the root is the last node.
 * `milliseconds` (optional) receives the build's wall time.  No counterpart
 * in the reference (whose builder, NexusBVH, is absent): it exposes the two
 * builders behind wf_scene_desc::bvh_builder for validation and timing. */
wf_status wf_bvh_build(uint32_t builder, const float* boxes, uint32_t count, uint32_t* nodes,
                       double* milliseconds);

/* ------------------------------------------------------- ray-level queries */
/* One ray: origin xyz, direction xyz (float). */
typedef struct wf_ray {
    float origin[3];
    float direction[3];
} wf_ray;

/* Closest hit of one ray, the fields of Hit (include/scene/geometry.cuh:68-82)
 * the shading stage uses plus the winning primitive's identity. */
typedef struct wf_hit {
    float t;
    float position[3];
    float geometric_normal[3];
    float normal[3];
    uint32_t material;    /* WF_NO_MATERIAL on a miss */
    uint32_t light_index; /* 0xffffffff when not a registered light */
    uint32_t kind;        /* WF_HIT_* */
    uint32_t instance;    /* instance index for WF_HIT_MESH, else 0xffffffff */
    uint32_t primitive;   /* sphere / triangle index within its list or mesh */
    float u, v;           /* barycentrics (triangles) */
} wf_hit;
enum { WF_HIT_NONE = 0, WF_HIT_MESH = 1, WF_HIT_STATIC_TRIANGLE = 2,
       WF_HIT_TRIANGLE = 3, WF_HIT_SPHERE = 4 };

/* Batched traceRay (device_traversal.cuh:1115-1184).  rays/hits are DEVICE
 * pointers; the call is asynchronous on `stream` (cudaStream_t, may be NULL). */
wf_status wf_trace_closest(const wf_scene* scene, const wf_ray* rays, uint32_t count,
                           wf_hit* hits, void* stream);
/* Batched isOccluded (device_traversal.cuh:1035-1113): occluded[i] = 1 when
 * something is hit at t < max_distance[i].  Device pointers, asynchronous. */
wf_status wf_trace_any(const wf_scene* scene, const wf_ray* rays, const float* max_distance,
                       uint32_t count, uint8_t* occluded, void* stream);

/* ------------------------------------------------------------------ render */
/* Camera, include/scene/camera.cuh:7-28 */
typedef struct wf_camera {
    float position[3];
    float forward[3];
    float right[3];
    float up[3];
    float vertical_fov; /* radians */
    float aspect_ratio;
} wf_camera;

/* FrameGuide (include/renderer/frame_guides.cuh:9-17), 56 bytes: the
 * denoiser guides of one pixel.  Normals are world space and face the
 * geometric normal's side; depth is the distance along the camera's forward
 * axis; motion is the previous frame's pixel minus this one (integer pixel
 * centres); valid = 1 on a hit; history_valid = 1 when the surface also
 * projects into the previous frame and is visible there. */
typedef struct wf_frame_guide {
    float albedo[3];
    float normal[3];
    float geometric_normal[3];
    float depth;
    float motion[2];
    float valid;
    float history_valid;
} wf_frame_guide;

/* generateFrameGuides (include/renderer/device_frame_guides.cuh:6-41) over
 * the tile (x, y, w, h) of a width x height image: one unjittered ray through
 * each pixel centre.  guides is a DEVICE array of w*h records, tile-local and
 * row-major, as tools/dataset_capture.cu:105-121 launches it.  previous (the
 * previous frame's camera) may be NULL: motion and history_valid stay 0.
 * Asynchronous on `stream` (cudaStream_t, may be NULL). */
wf_status wf_frame_guides(const wf_scene* scene, const wf_camera* camera, const wf_camera* previous,
                          uint32_t width, uint32_t height, uint32_t x, uint32_t y, uint32_t w, uint32_t h,
                          wf_frame_guide* guides, void* stream);

/* GRAPH: the reference's captured wavefront, one graph replay per tile and
 * sample (render_driver.cu:264-352).  PERSISTENT: one cooperative launch per
 * tile and sample (renderer.cu:55-125).  STREAM: one graph replay per tile
 * covers the whole sample range; a slot whose path ends starts the same
 * pixel's next sample in the same loop iteration (a device-side while loop,
 * so the short tail bounces of many samples share launches).  Each pixel
 * still adds its samples to the framebuffer one after another in sample
 * order, so the three modes give bit-identical framebuffers. */
enum { WF_MODE_GRAPH = 0, WF_MODE_PERSISTENT = 1, WF_MODE_STREAM = 2 };
enum { WF_RNG_XORSHIFT32 = 0, WF_RNG_PCG32 = 1 };
enum { WF_DEBUG_NONE = 0, WF_DEBUG_INTERSECTION = 1, WF_DEBUG_SHADING_NORMAL = 2 };

/* RenderConfig, include/config.hpp:11-41 (the fields the render loop reads). */
typedef struct wf_render_config {
    uint32_t width, height;
    uint32_t max_depth;
    uint32_t rr_start_depth;
    uint32_t mode;             /* WF_MODE_* */
    uint32_t rng;              /* WF_RNG_* */
    float indirect_clamp;      /* 0 disables */
    uint32_t tile_width;       /* 0 = full frame; bounds queue memory */
    uint32_t tile_height;
    uint32_t block_size;       /* CTA size of the lane-refill trace and shadow kernels: a multiple of
                                  32 up to 1024; 0 = 128 */
    uint32_t persistent_blocks;/* 0 = the resident grid, trimmed for small tiles to
                                  max(4 x SMs, paths / 128) */
    uint32_t chunk;            /* persistent work chunk in paths, 0 = default */
    uint32_t debug;            /* WF_DEBUG_* */
    /* photon caustics, src/renderer/photon_mapping.cu + render_driver.cu:180-234 */
    uint32_t caustics;
    uint32_t caustic_gather;
    uint32_t photon_count;
    uint32_t photon_max_depth;
    float gather_radius;
    float photon_grid_min[3];  /* grid bounds; min == max derives them from the scene */
    float photon_grid_max[3];
    uint32_t photon_grid_resolution;
    uint32_t photon_seed;
    uint32_t spectral;
    uint32_t profile_queues;   /* record per-bounce queue counts */
    uint32_t refill_threshold; /* trace/shadow kernels: a warp fetches new rays once this many of its
                                  lanes are idle (1..32; 0 = default 8) */
    uint32_t concurrent_tiles; /* graph mode: 2 (or 0 = default) = two wavefronts on two streams, each
                                  rendering its own rows of every tile, so the long last bounces of one
                                  overlap the other's work; 1 = one wavefront.  Each pixel stays with one
                                  wavefront, so the sums are the same either way. */
    uint32_t shadow_queue_capacity; /* graph and streaming modes: shadow-ray requests one bounce can
                                  queue; 0 = (5 + directional lights) x queue slots, which no bounce
                                  can exceed.  Requests beyond a smaller capacity are dropped (their
                                  terms count as unoccluded) and wf_synchronize reports
                                  WF_ERR_CAPACITY, as the reference's bounded appendWarpCompacted
                                  drops items beyond a queue's capacity (queue_compaction.cuh:8-29). */
    uint32_t regenerate_percent; /* streaming mode: a slot whose path ended starts its pixel's next sample
                                  once fewer than this percentage of the tile's slots still carry a
                                  path; all waiting slots then start together, in slot order, and
                                  their camera rays are traced coherently.  1..100 (100 = after every
                                  bounce); 0 = the tuned default.  Each pixel still takes its samples
                                  in order, so the sums do not depend on it. */
    uint32_t persistent_stages; /* persistent mode: WF_PERSISTENT_AUTO (0) = staged from 262,144 paths
                                  per tile, fused below; WF_PERSISTENT_FUSED = one body per path
                                  (trace, shade, shadow rays inline, as persistentWavefrontTrace);
                                  WF_PERSISTENT_STAGED = the wavefront stages between grid barriers.
                                  Same sums either way. */
    uint32_t samples_per_wave; /* graph mode and the staged persistent kernel: samples of every pixel
                                  of the tile that one launch traces together (0 or 1 = one, as the
                                  reference's per-sample replay; at most 1024; in persistent mode a
                                  wave above 1 selects the staged kernel unless persistent_stages is
                                  WF_PERSISTENT_FUSED, which ignores it).  The long last bounces of these
                                  samples then share one chain of launches.  Each path's radiance is
                                  added to the framebuffer after the launch, per pixel in sample
                                  order, so the sums do not depend on it; queue memory grows with it,
                                  and wf_queue_counts reports the counts of the whole launch. */
} wf_render_config;
enum { WF_PERSISTENT_AUTO = 0, WF_PERSISTENT_FUSED = 1, WF_PERSISTENT_STAGED = 2 };

/* Defaults of RenderConfig (config.hpp:11-41) at the given resolution. */
void wf_render_config_default(wf_render_config* config, uint32_t width, uint32_t height);

typedef struct wf_renderer wf_renderer;

/* Replaces RenderDriver(const DeviceScene&, Camera, RenderConfig, SceneConfig)
 * + RenderDriver::prepare (render_driver.cu:422-449): validates the config,
 * sizes the persistent grid, builds the photon map, allocates queues and
 * captures the bounce chain into a CUDA graph (graph mode).
 * `stream` is a cudaStream_t (NULL = renderer-owned non-blocking stream). */
wf_status wf_renderer_create(const wf_scene* scene, const wf_camera* camera,
                             const wf_render_config* config, void* stream,
                             wf_renderer** out);
wf_status wf_renderer_destroy(wf_renderer* renderer);

/* Replaces RenderTaskRenderer::render(const RenderTask&), render_task.cu:26-114:
 * renders absolute samples [sample_start, sample_start + sample_count) of the
 * tile.  clear_tile = 1 zeroes the tile first (the task semantics: the tile
 * then holds the unnormalized sum over the range); 0 accumulates.
 * Asynchronous on the renderer stream. */
wf_status wf_render(wf_renderer* renderer, uint32_t x, uint32_t y, uint32_t width,
                    uint32_t height, uint32_t sample_start, uint32_t sample_count,
                    uint32_t clear_tile);
/* Replaces RenderDriver::renderSamples (render_driver.cu:354-401): renders
 * sample_count samples over all tiles, continuing from the device sample
 * index, which advances by one per sample.  Asynchronous. */
wf_status wf_render_frame(wf_renderer* renderer, uint32_t sample_count);

/* resetRenderSession / setRenderSessionSampleIndex / getRenderSessionSampleIndex,
 * src/renderer/render_session.cu:28-42 */
wf_status wf_framebuffer_reset(wf_renderer* renderer);
wf_status wf_set_sample_index(wf_renderer* renderer, uint32_t sample_index);
wf_status wf_get_sample_index(wf_renderer* renderer, uint32_t* sample_index);
/* Copies the unnormalized FP32 RGB sums of a tile (row-major, 3 floats per
 * pixel) into host memory; synchronizes the stream.  (cudaMemcpy2D of
 * render_task.cu:101-108.) */
wf_status wf_framebuffer_download(wf_renderer* renderer, uint32_t x, uint32_t y,
                                  uint32_t width, uint32_t height, float* rgb);
/* Starts the copy of a tile's sums into host memory, as
 * wf_framebuffer_download does, and returns without waiting.  The renderer
 * first snapshots the tile on the device in stream order, so the wf_render
 * calls made after this one run while the snapshot crosses PCIe (with
 * page-locked `rgb` memory; pageable memory works, without the overlap).
 * Two copies may be in flight; a third waits on the device for the oldest.
 * `rgb` holds the data once wf_framebuffer_download_wait or wf_synchronize
 * has returned.  The reference overlaps its checkpoint copies with
 * rendering in the same way (enqueueAsyncCheckpoint, render_session.cuh:
 * 22-26).  The first call allocates two framebuffer-sized device
 * snapshots. */
wf_status wf_framebuffer_download_async(wf_renderer* renderer, uint32_t x, uint32_t y,
                                        uint32_t width, uint32_t height, float* rgb);
/* Waits until every copy started by wf_framebuffer_download_async has
 * arrived; work issued on the renderer's stream afterwards is ordered after
 * those copies. */
wf_status wf_framebuffer_download_wait(wf_renderer* renderer);
/* Device address of the width*height*3 float framebuffer. */
wf_status wf_framebuffer_device(wf_renderer* renderer, float** rgb);
/* Waits for the renderer's work and reports the errors its kernels recorded:
 * WF_ERR_TIMEOUT when a bounded wait gave up (a persistent-kernel grid
 * barrier, or the streaming loop's iteration bound), WF_ERR_CAPACITY when a
 * queue overflowed.  The reference exits the process on device errors
 * (render_driver.cu:18-27); here the flags are cleared once reported, so the
 * renderer stays usable and the next call renders correctly. */
wf_status wf_synchronize(wf_renderer* renderer);

/* Bounds of the renderer's device-side waits (no counterpart in the
 * reference).  barrier_cycles: clock cycles a persistent-kernel grid barrier
 * waits for the other blocks before it gives up (0 = 2^31).
 * loop_iterations: passes of the streaming schedule's device-side loop per
 * launch (0 = the bound samples x max_depth / 2 + 1 that no correct render
 * reaches).  Smaller values let a watchdog (or a test) make the waits run
 * out; the render then reports WF_ERR_TIMEOUT from wf_synchronize.
 * Stream-ordered: applies to work queued after the call. */
wf_status wf_renderer_set_watchdog(wf_renderer* renderer, uint64_t barrier_cycles, uint32_t loop_iterations);

/* Per-bounce ray-queue sizes of the most recent sample of the most recent
 * tile (the --profile-queues record, renderer.cu:89-90).  Requires
 * profile_queues; writes min(n, max_depth) counts. */
wf_status wf_queue_counts(wf_renderer* renderer, uint32_t* counts, uint32_t n);

typedef struct wf_render_stats {
    uint64_t extension_rays;
    uint64_t shadow_rays;
    uint64_t paths;
    uint64_t kernel_launches;  /* render-kernel launches that ran (device-counted) */
} wf_render_stats;
/* Ray counters accumulated since creation or the last reset (synchronizes). */
wf_status wf_render_stats_get(wf_renderer* renderer, wf_render_stats* stats, uint32_t reset);

/* Persistent-mode render of one tile that allocates no device memory.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc while rendering (a host embedded in another framework's memory
 * pool, a process whose device-memory budget is fixed at start-up, or code
 * that must not trigger the implicit synchronization an allocation can
 * cause).  The caller owns the scene and `framebuffer` (a DEVICE buffer of
 * config->width * config->height * 3 floats, already zeroed or holding
 * earlier sums); the call ADDS the unnormalized sums of samples
 * [sample_start, sample_start + sample_count) of pixels inside the tile,
 * exactly as wf_render with WF_MODE_PERSISTENT does.  Working memory is one
 * fixed 6.3 MB device array inside the library that every GPU loading the
 * library holds until the process exits; tiles above 65,536 pixels return
 * WF_ERR_CAPACITY and configs with caustics return WF_ERR_UNSUPPORTED.
 * The first call on each device looks up the array's device address and the
 * kernel's resident grid (no allocation); a device whose context was
 * re-created (cudaDeviceReset) gets the same set-up again on its next call.
 * Every call shares the one array (it is reset at the start of each call):
 * calls whose GPU work overlaps, from several host threads or streams, race
 * and give wrong images.  The call returns after the work on
 * `stream` (cudaStream_t, may be NULL) has finished. */
wf_status wf_render_tile_static(const wf_scene* scene, const wf_camera* camera,
                                const wf_render_config* config, uint32_t x, uint32_t y,
                                uint32_t width, uint32_t height, uint32_t sample_start,
                                uint32_t sample_count, float* framebuffer, void* stream);

/* Candidate settings of wf_renderer_autotune.  Each list comes with its
 * length; a length of 0 keeps the base config's value.  Settings that a mode
 * does not read are not varied for it (concurrent_tiles: graph mode only;
 * regenerate_percents: streaming mode only; persistent_stages: persistent
 * mode only, with chunks varied for its fused kernel only). */
typedef struct wf_tune_space {
    const uint32_t* modes;               uint32_t mode_count;               /* WF_MODE_* */
    const uint32_t* block_sizes;         uint32_t block_size_count;         /* trace / shade CTA size */
    const uint32_t* refill_thresholds;   uint32_t refill_threshold_count;   /* lane refill (1..32) */
    const uint32_t* concurrent_tiles;    uint32_t concurrent_tiles_count;   /* wavefronts per tile */
    const uint32_t* regenerate_percents; uint32_t regenerate_percent_count; /* streaming regeneration */
    const uint32_t* chunks;              uint32_t chunk_count;              /* persistent work chunk (fused) */
    const uint32_t* persistent_stages;   uint32_t persistent_stage_count;   /* WF_PERSISTENT_* */
    const uint32_t* tile_sizes;          uint32_t tile_size_count;          /* square tile edge = queue
                                                                               capacity; 0 = full frame */
    uint32_t samples;  /* samples per pixel of each timed frame (0 = 1) */
    const uint32_t* samples_per_waves;   uint32_t samples_per_wave_count;   /* graph mode: samples per wave */
} wf_tune_space;

/* Single-scene autotuner (no counterpart in the reference, whose block size
 * and schedule are fixed settings of config.hpp).  For every combination of
 * the candidate settings it creates a renderer from `base` (same scene,
 * camera and image), renders one untimed frame of space->samples samples per
 * pixel, then one timed frame (CUDA events on the renderer stream), and
 * keeps the fastest.  `best` receives that config; times_ms[i] (optional,
 * times_capacity entries) the frame time of candidate i in loop order
 * (modes outermost, then block sizes, refill thresholds, tile sizes, and the
 * mode's own settings: concurrent tiles, each by samples per wave;
 * regenerate percents; persistent stages, each fused one by chunk);
 * *evaluated the number of candidates.  A candidate whose buffers do not
 * fit in device memory is skipped (its time is +inf; WF_ERR_OOM when none
 * fits).  All candidates
 * render the same image, so the choice does not change any result. */
wf_status wf_renderer_autotune(const wf_scene* scene, const wf_camera* camera, const wf_render_config* base,
                               const wf_tune_space* space, void* stream, wf_render_config* best,
                               float* times_ms, uint32_t times_capacity, uint32_t* evaluated);

/* Kernel-level profile of one pass over the whole frame (one wave of
 * samples_per_wave samples in graph mode, one sample otherwise). */
enum { WF_KERNEL_RAYGEN = 0, WF_KERNEL_TRACE = 1, WF_KERNEL_SHADE = 2, WF_KERNEL_SHADOW = 3,
       WF_KERNEL_FINALIZE = 4, WF_KERNEL_PERSISTENT = 5, WF_KERNEL_GATHER = 6, WF_KERNEL_KINDS = 7 };
enum { WF_PROFILE_BOUNCES = 32 };
typedef struct wf_kernel_profile {
    uint32_t launches[WF_KERNEL_KINDS];
    float milliseconds[WF_KERNEL_KINDS];   /* summed CUDA-event durations */
    uint64_t extension_rays;
    uint64_t shadow_rays;
    /* traversal work of the pass: closest-hit kernel, then shadow kernel */
    uint64_t closest_nodes, closest_triangles, closest_spheres, closest_instances;
    uint64_t any_nodes, any_triangles, any_spheres, any_instances;
    /* graph mode, per bounce of the timing replay summed over tiles: event
     * times of trace, shade, shadow, finalize and caustic gather, extension
     * rays traced and shadow rays requested (bounces >= WF_PROFILE_BOUNCES
     * are not split) */
    float bounce_milliseconds[5][WF_PROFILE_BOUNCES];
    uint32_t bounce_extension_rays[WF_PROFILE_BOUNCES];
    uint32_t bounce_shadow_rays[WF_PROFILE_BOUNCES];
} wf_kernel_profile;
/* Renders one more pass (a wave in graph mode) over all tiles with every
 * kernel launched eagerly and bracketed by CUDA events on the renderer
 * stream (the timing replay), then one more with counting traversal kernels
 * (the work tally).  Both passes accumulate into the framebuffer.
 * Supplements the reference's --profile-queues record (render_driver.cu:393-400). */
wf_status wf_profile_sample(wf_renderer* renderer, wf_kernel_profile* profile);

/* Photon map (buildPhotonMap, render_driver.cu:180-234): number of photons
 * stored on diffuse surfaces after >= 1 specular bounce. */
wf_status wf_photon_stats(wf_renderer* renderer, uint32_t* stored, uint32_t* emitted);
/* Downloads photon records as 8 floats each: position xyz, direction xyz,
 * flux sum, valid flag (host memory, count = emitted). */
wf_status wf_photons_download(wf_renderer* renderer, float* records, uint32_t count);

/* ------------------------------------------------------------------- batch */
/* Many independent render jobs (own scene, camera, resolution, depth and
 * sample range) in one captured graph.  No counterpart in the reference,
 * which renders one job per RenderDriver.  A pool of path slots works
 * through (job, pixel) units; a slot renders all of its unit's samples in
 * sample order before it takes the next unit, so each job's framebuffer is
 * bit-identical to a wf_render of that job's sample range.  Caustics are
 * not supported in a batch (WF_ERR_UNSUPPORTED). */
typedef struct wf_batch wf_batch;
typedef struct wf_batch_job {
    const wf_scene* scene;
    wf_camera camera;
    wf_render_config config;   /* width/height = the job's image; mode and tile fields are ignored */
    uint32_t sample_start;     /* absolute first sample */
    uint32_t sample_count;
} wf_batch_job;
typedef struct wf_batch_config {
    uint32_t slot_capacity;    /* paths in flight; 0 = min(paths of a pass, 4M) */
    uint32_t block_size;       /* trace/shade/shadow CTA size; 0 = 128 */
    uint32_t refill_threshold; /* as in wf_render_config; 0 = 8 */
    uint32_t longest_first;    /* 1 = start the jobs with the most samples x depth per pixel first */
    uint32_t pass_paths;       /* paths (pixel samples) per pass, each holding a 16-byte radiance
                                  record until its pixel adds it; 0 = 2^27 (2 GB) */
} wf_batch_config;
void wf_batch_config_default(wf_batch_config* config);
wf_status wf_batch_create(const wf_batch_job* jobs, uint32_t job_count, const wf_batch_config* config,
                          void* stream, wf_batch** out);
/* Renders every job's sample range once (one graph launch per pass of
 * pass_paths paths; asynchronous on the batch stream), adding to the job
 * framebuffers: each pixel adds its samples in sample order after the pass
 * that traced them, so every framebuffer equals a per-job wf_render's.
 * A batch holds fewer than 2^32 paths. */
wf_status wf_batch_run(wf_batch* batch);
wf_status wf_batch_synchronize(wf_batch* batch);
wf_status wf_batch_reset(wf_batch* batch);   /* zero every job framebuffer */
/* Job framebuffer, width * height * 3 floats (host copy; synchronizes). */
wf_status wf_batch_download(wf_batch* batch, uint32_t job, float* rgb);
wf_status wf_batch_framebuffer_device(wf_batch* batch, uint32_t job, float** rgb);
wf_status wf_batch_stats(wf_batch* batch, wf_render_stats* stats, uint32_t reset);
wf_status wf_batch_destroy(wf_batch* batch);

/* Autotuner: renders the batch once per candidate (slot capacity x block
 * size x refill threshold; zero-terminated lists, NULL = defaults), times
 * each run with CUDA events and writes the fastest configuration to *best.
 * times_ms (optional) receives one entry per candidate in list order. */
wf_status wf_batch_autotune(const wf_batch_job* jobs, uint32_t job_count, const uint32_t* slot_capacities,
                            const uint32_t* block_sizes, const uint32_t* refill_thresholds, void* stream,
                            wf_batch_config* best, float* times_ms, uint32_t times_capacity);

/* ----------------------------------------------------------- differentiable */
/* Path-replay adjoint renderer (no counterpart in the reference).  Its own
 * material model: every non-emissive triangle has an Oren-Nayar BRDF with
 * RGB albedo and roughness (radians) read from caller arrays indexed by the
 * triangle's index in its mesh or triangle list; emissive materials emit
 * emission * emission_scale.  Next-event estimation over the triangle
 * lights, cosine-sampled continuations, no Russian roulette, no clamp.
 * image = emission_scale / spp * sum of path radiance (RGB floats, full
 * width x height layout; only the crop is written).  Sampling never depends
 * on the parameters, so wf_diff_backward returns, for each path, the exact
 * derivative of its estimate: it replays each path from its RNG key (no
 * path storage, memory O(pixels)) and ADDS dLoss/dparameter to the double
 * gradient arrays.  All pointers are device pointers; both calls
 * synchronize `stream`. */
typedef struct wf_diff_config {
    uint32_t width, height;     /* image (camera aspect and pixel RNG index) */
    uint32_t crop_x, crop_y, crop_width, crop_height;  /* 0 width/height = whole image */
    uint32_t spp;
    uint32_t sample_start;      /* absolute first sample */
    uint32_t max_depth;         /* path vertices */
    uint32_t rng;               /* WF_RNG_* */
    uint32_t parameter_count;   /* triangles with parameters (albedo has 3 x this many floats) */
} wf_diff_config;
wf_status wf_diff_forward(const wf_scene* scene, const wf_camera* camera, const wf_diff_config* config,
                          const float* albedo, const float* roughness, float emission_scale, float* image,
                          void* stream);
wf_status wf_diff_backward(const wf_scene* scene, const wf_camera* camera, const wf_diff_config* config,
                           const float* albedo, const float* roughness, float emission_scale,
                           const float* d_image, double* d_albedo, double* d_roughness,
                           double* d_emission_scale, void* stream);
/* Albedo gradients of the renderer's own image (no counterpart in the
 * reference).  Replays samples [sample_start, sample_start + sample_count)
 * of the pixels of the tile (x, y, width, height) with the renderer's
 * shading, and ADDS to gradient[3*m .. 3*m+2] the derivative of
 * sum over pixels and channels of adjoint * (sum of the samples' radiance)
 * with respect to the RGB albedo of materials[m].  The random numbers are
 * those wf_render draws, and Russian roulette's 1/survival weight is held
 * constant: the result is the exact derivative of each sample's estimate
 * for the survival decisions it drew (exact outright when rr_start_depth
 * >= max_depth), an unbiased estimate of the gradient of the expected
 * image.  When `image` is not null the replay also writes the tile's
 * sample sums there, bit for bit the framebuffer wf_render leaves after
 * rendering the same samples from a cleared framebuffer.  The parameter
 * materials (1 to 8, distinct) must be untextured, non-metallic diffuse
 * materials with non-zero albedo; the renderer must have caustics off,
 * indirect_clamp 0 and no debug view (WF_ERR_UNSUPPORTED otherwise).
 * `materials` is a host array; adjoint, image and gradient are device
 * arrays (adjoint and image full width x height x 3 floats).  Runs on the
 * renderer's stream and synchronizes it. */
wf_status wf_render_albedo_gradient(wf_renderer* renderer, uint32_t x, uint32_t y, uint32_t width,
                                    uint32_t height, uint32_t sample_start, uint32_t sample_count,
                                    const uint32_t* materials, uint32_t material_count, const float* adjoint,
                                    float* image, double* gradient);

/* -------------------------------------------------------------- checkpoint */
/* Checkpoint file: header {magic "PTCHKPT1", version 3, width, height,
 * sampleIndex, fingerprint} + width*height Vec3 (render_checkpoint.cpp:17-63).
 * wf_checkpoint_save writes via a temporary file and rename. */
wf_status wf_checkpoint_save(wf_renderer* renderer, const char* path, uint64_t fingerprint);
/* Asynchronous variant (enqueueRenderSessionCheckpoint, render_checkpoint.cpp:108-138):
 * copies the framebuffer into one of `slots` pinned buffers on the render
 * stream and writes it from a worker thread.  *queued = 0 when every slot is
 * busy (the checkpoint is skipped, as the reference does). */
wf_status wf_checkpoint_enqueue(wf_renderer* renderer, const char* path, uint64_t fingerprint,
                                uint32_t* queued);
/* Waits for queued checkpoint writes (finishAsyncCheckpointWriter). */
wf_status wf_checkpoint_flush(wf_renderer* renderer);
/* Replaces loadRenderSessionCheckpoint (render_checkpoint.cpp:163-195); returns
 * WF_ERR_FORMAT / WF_ERR_FINGERPRINT / WF_ERR_IO instead of exiting. */
wf_status wf_checkpoint_load(wf_renderer* renderer, const char* path, uint64_t fingerprint,
                             uint32_t* sample_index);
/* FNV-1a 64 over bytes (the hash of render_fingerprint.cpp:11-83). */
uint64_t wf_fnv1a64(const void* data, size_t size, uint64_t seed);

#ifdef __cplusplus
}
#endif

#endif /* WAVEFRONT_H */
