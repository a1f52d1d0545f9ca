// Host-side structures of the renderer runtime (not part of the C ABI).
#pragma once

#include <cstdarg>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/wavefront.h"
#include "bvh_build.h"
#include "wf_device.cuh"

namespace wf {

// Records the thread-local error text returned by wf_last_error().
wf_status fail(wf_status status, const char* format, ...);

// Every device allocation of the library goes through device_alloc, so a
// test can make one of them fail (wf_test_fail_allocation) and check that
// the entry point frees what it allocated and reports WF_ERR_OOM.
cudaError_t device_alloc(void** p, size_t bytes);

// The scene after the host build, in device layout (see wf_device.cuh).
struct HostScene {
    std::vector<float4> triangles;  // 3 per triangle
    std::vector<float4> normals;    // 3 per triangle when any triangle has vertex normals
    std::vector<BvhNode> nodes;
    std::vector<Blas> blases;
    std::vector<Instance> instances;
    std::vector<uint32_t> mesh_linear;
    std::vector<uint32_t> tlas_leaves;
    std::vector<float4> spheres;
    std::vector<uint32_t> sphere_materials;
    std::vector<uint32_t> direct_spheres;
    std::vector<uint32_t> direct_instances;
    std::vector<Material> materials;
    std::vector<MaterialTextures> material_textures;  // empty without texture bindings
    std::vector<uchar4> texels;
    std::vector<uint4> textures;
    std::vector<TriAttr> tri_attr;                    // empty without triangle attributes
    bool use_normal_maps = true;
    float normal_map_min_cosine = 0.0f;
    std::vector<Light> lights;
    std::vector<Punctual> punctual;
    uint32_t directional_count = 0;
    BvhRef tlas{kNoRoot, {}};
    BvhRef direct_bvh{kNoRoot, {}};
    uint32_t static_first = 0, static_count = 0;
    uint32_t direct_first = 0, direct_count = 0;
    bool any_alpha_reject = false;
    bool black_background = false;
    bool ignore_occlusion = false;
    Box bounds{};  // world bounds of all geometry (photon-grid default)
    uint32_t gpu_bvh_builds = 0;
    double bvh_build_ms = 0.0;
    bool alpha_textures = false;
    bool textured = false;
};

// Builds the device-layout scene: light registration, light alias table,
// BLAS/TLAS/direct BVHs, packing.  Restates src/scene/scene.cu:82-294,336-389
// and src/scene/scene_host.cpp:60-106.
wf_status build_host_scene(const wf_scene_desc* desc, HostScene& out);

struct HostEnvironment {
    uint32_t width = 0, height = 0;
    std::vector<float4> pixels;
    std::vector<float> probabilities;
    std::vector<float2> alias;
    std::vector<float> row_solid_angle;
    float intensity = 1.0f;
    float rotation = 0.0f;
};

// buildEnvironmentDistribution (src/scene/environment.cpp:10-64) plus the
// uploadEnvironmentMap validation and rotation (src/scene/scene.cu:308-334).
wf_status build_environment(const wf_environment* env, HostEnvironment& out);

// environmentSolidAngle, include/scene/environment.cuh:35-39.
float environment_solid_angle(uint32_t row, uint32_t width, uint32_t height);

}  // namespace wf

// Opaque C-ABI scene: device buffers plus the kernel view.
struct wf_scene {
    wf::DeviceScene view{};
    std::vector<void*> allocations;
    std::vector<void*> env_allocations;
    uint64_t device_bytes = 0;
    uint64_t env_bytes = 0;
    uint32_t light_count = 0;
    uint32_t tlas_leaf_count = 0;
    uint32_t blas_count = 0;
    uint32_t material_count = 0;
    double build_seconds = 0.0;
    uint32_t gpu_bvh_builds = 0;
    double bvh_build_ms = 0.0;
    bool alpha_textures = false;  // some material is alpha-masked with an albedo texture
    bool textured = false;        // some material has a texture binding
    uint32_t material_categories = 0;  // bit k: some material has shading category k (material_category)
    wf::Box bounds{};
    int device = 0;
};
