// Device-side scene layout and vector arithmetic of the B200 renderer.
//
// Layout (all arrays in HBM, read through the read-only path):
//   * triangles: 3 x float4 per triangle (48 B, one 16-byte-aligned load per
//     vertex).  .w lanes carry the original index | flags, the material and
//     the light index.  Every mesh, the static list and the direct list share
//     one array; BLAS leaves reference triangles in leaf order so a subtree's
//     triangles are contiguous.
//   * BVH2 nodes: 64 B, both child boxes stored in the parent
//     (lxy | rxy | lrz | children), so one node visit is four 16-byte loads and
//     tests two boxes.  Child refs >= 0 are node indices, < 0 are ~leaf.
//   * spheres: float4 (center, radius) + material.
// The arithmetic helpers reproduce the reference's Vec3 operators
// (include/core/vec3.cuh:6-99) operation for operation so that, compiled with
// -fmad=false, results match an IEEE host build of the reference bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "wf_math.h"

#if defined(__CUDACC__)
#define WF_DEV __device__ __forceinline__
#define WF_HDI __host__ __device__ __forceinline__
// Large shading helpers called from several sites: one out-of-line copy.
#define WF_CALL static __device__ __noinline__
#else
#define WF_DEV inline
#define WF_HDI inline
#define WF_CALL inline
#endif

namespace wf {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr float kRayMinDistance = 1.0e-6f;  // include/core/ray.cuh:8

// ----------------------------------------------------------------- vectors
struct V3 {
    float x, y, z;
};
WF_HDI V3 v3(float x, float y, float z) { return V3{x, y, z}; }
WF_HDI V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
WF_HDI V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
WF_HDI V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
WF_HDI V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
WF_HDI V3 operator*(float s, V3 a) { return a * s; }
// vec3.cuh:45-48: division multiplies by the reciprocal.
WF_HDI V3 operator/(V3 a, float s) {
    float inv = 1.0f / s;
    return a * inv;
}
WF_HDI V3& operator+=(V3& a, V3 b) {
    a.x += b.x; a.y += b.y; a.z += b.z;
    return a;
}
WF_HDI V3& operator*=(V3& a, float s) {
    a.x *= s; a.y *= s; a.z *= s;
    return a;
}
WF_HDI float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
WF_HDI V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
WF_HDI float length_squared(V3 v) { return dot(v, v); }
WF_HDI float length(V3 v) { return sqrtf(length_squared(v)); }
WF_HDI V3 normalize(V3 v) {
    float inv = 1.0f / sqrtf(dot(v, v));
    return v * inv;
}
WF_HDI V3 hadamard(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
WF_HDI V3 f4xyz(float4 f) { return V3{f.x, f.y, f.z}; }

// offsetRayOrigin, include/core/ray.cuh:10-21.
WF_HDI V3 offset_ray_origin(V3 position, V3 normal, V3 direction, float hit_distance) {
    float magnitude = fmaxf(fmaxf(1.0f, fabsf(hit_distance)),
                            fmaxf(fabsf(position.x), fmaxf(fabsf(position.y), fabsf(position.z))));
    float sign = dot(direction, normal) >= 0.0f ? 1.0f : -1.0f;
    V3 offset = normal * (sign * 32.0f * 1.1920928955078125e-7f * magnitude);
    V3 result = position + offset;
    if (offset.x != 0) result.x = nextafterf(result.x, offset.x > 0 ? INFINITY : -INFINITY);
    if (offset.y != 0) result.y = nextafterf(result.y, offset.y > 0 ? INFINITY : -INFINITY);
    if (offset.z != 0) result.z = nextafterf(result.z, offset.z > 0 ? INFINITY : -INFINITY);
    return result;
}

// ------------------------------------------------------------------ layout
struct alignas(16) BvhNode {
    float4 lxy;  // left  lo.x, hi.x, lo.y, hi.y
    float4 rxy;  // right lo.x, hi.x, lo.y, hi.y
    float4 lrz;  // left lo.z, hi.z, right lo.z, hi.z
    int4 child;  // x = left ref, y = right ref (>= 0 node, < 0 ~leaf)
};
static_assert(sizeof(BvhNode) == 64, "BVH node must be 64 bytes");

struct Box {
    float lo[3];
    float hi[3];
};

// One BVH: root ref (node index, or ~leaf when the tree is a single leaf,
// or kNoRoot when empty) and the root box.
constexpr int kNoRoot = 0x7fffffff;
struct BvhRef {
    int root;
    Box box;
};

// Triangle .w lanes: a.w = original index | kTriHasNormals, b.w = material,
// c.w = light index.
constexpr uint32_t kTriHasNormals = 0x80000000u;
constexpr uint32_t kTriIndexMask = 0x7fffffffu;

struct Blas {
    BvhRef bvh;            // bvh.root == kNoRoot when built without BVH
    uint32_t first;        // first triangle (leaf order) in the global array
    uint32_t count;
    uint32_t first_linear; // offset into mesh_linear (original order)
};

struct Instance {
    float4 w2l_x;  // worldToLocalX.xyz, translation.x
    float4 w2l_y;  // worldToLocalY.xyz, translation.y
    float4 w2l_z;  // worldToLocalZ.xyz, translation.z
    float4 l2w_x;  // localToWorldX.xyz, (unused)
    float4 l2w_y;
    float4 l2w_z;
    uint32_t blas;
    uint32_t light_offset;
    uint32_t material_override;
    uint32_t pad;
};

// Material flags.
constexpr uint32_t kMatGltfPbr = 1u;
constexpr uint32_t kMatSpecGlossWorkflow = 2u;
constexpr uint32_t kMatAlphaReject = 4u;  // alphaMasked && opacity < alphaCutoff (untextured)
constexpr uint32_t kMatTextured = 8u;      // some texture binding is set: resolve factors at the hit
constexpr uint32_t kMatAlphaTexture = 16u; // alphaMasked with an albedo texture: opacity per hit

// Untextured Material (include/scene/material.cuh:30-70): every texture
// lookup returns its factor, so only the factors are kept.
struct Material {
    uint32_t type;
    uint32_t flags;
    float roughness, ior;
    V3 albedo;
    V3 emission;
    float metallic, dispersion;
    V3 attenuation_color;
    float attenuation_distance;
    float volume_density;
    float glossiness;
    V3 specular;
    float specular_weight;
    V3 specular_color;
    float clearcoat;
    float clearcoat_roughness;
};

enum MaterialType : uint32_t { kDiffuse = 0, kMetal = 1, kDielectric = 2, kEmissive = 3, kSpecGloss = 4 };

// Shading categories (the key of the material sort before shading):
// 0 miss, 1 emissive, 2 diffuse, 3 metal, 4 dielectric, 5 other.
constexpr uint32_t kShadeCategories = 6;
WF_HDI uint32_t material_category(const Material& mat) {
    if (mat.flags & kMatGltfPbr) return 5;
    switch (mat.type) {
    case kEmissive: return 1;
    case kDiffuse: return mat.metallic > 0.5f ? 3 : 2;
    case kMetal: return 3;
    case kDielectric: return 4;
    default: return 5;
    }
}

// TextureBinding, include/scene/material.cuh:14-21.
struct TexBinding {
    uint32_t texture;  // kInvalid: none
    uint32_t texcoord;
    float offset_x, offset_y, scale_x, scale_y, rotation;
    uint32_t has_transform;
};

enum TexSlot : uint32_t {
    kTexAlbedo = 0,
    kTexMetallicRoughness,
    kTexEmissive,
    kTexNormal,
    kTexThickness,
    kTexSpecGloss,
    kTexSpecularWeight,
    kTexSpecularColor,
    kTexClearcoat,
    kTexClearcoatRoughness,
    kTexClearcoatNormal,
    kTexSlots
};

// The texture side of a Material (include/scene/material.cuh:42-69), read
// only for materials flagged kMatTextured / kMatAlphaTexture.
struct MaterialTextures {
    float normal_scale, clearcoat_normal_scale;
    float opacity, alpha_cutoff;
    TexBinding slot[kTexSlots];
};

// Texture coordinates and tangent frames of one triangle
// (include/scene/geometry.cuh:22-41), in triangle packing order.
struct TriAttr {
    float uv[3][2];
    float uv1[3][2];
    float tangent[3], bitangent[3], tangent1[3], bitangent1[3];
    float vertex_tangent[3][3];
    float vertex_tangent_sign[3];
    uint32_t has_vertex_tangents;
    uint32_t has_texcoords;
    uint32_t has_texcoords1;
    uint32_t pad;
};
static_assert(sizeof(TriAttr) == 160, "TriAttr is 40 words");

// TriangleLight, include/scene/geometry.cuh:49-57.
struct Light {
    V3 v0, v1, v2, normal;
    float area;
    uint32_t material;
    float selection_pdf;
    float alias_probability;
    uint32_t alias;
    uint32_t pad[3];
};

// PunctualLight, include/scene/punctual_light.cuh:8-16.
struct Punctual {
    uint32_t type;
    V3 position, direction, intensity;
    float range, inner_cone_cos, outer_cone_cos;
};

struct Environment {
    const float4* pixels;
    const float* probabilities;
    const float2* alias;           // (probability, alias index bits)
    const float* row_solid_angle;  // environmentSolidAngle(row), environment.cuh:35-39
    uint32_t width, height;
    float intensity;
    float rotation;
    float cos_rot, sin_rot;        // cosf/sinf(rotation)
    float cos_neg, sin_neg;        // cosf/sinf(-rotation)
    uint32_t present;              // texture bound (EnvironmentView::texture != 0)
    uint32_t sampling;             // diffuseEnvironmentProbability() > 0
};

// Hit kinds stored in the top two bits of a hit's primitive word.
constexpr uint32_t kHitMiss = 0u;
constexpr uint32_t kHitMesh = 1u;      // triangle of an instance (instance word valid)
constexpr uint32_t kHitTriangle = 2u;  // world-space triangle (static or direct list)
constexpr uint32_t kHitSphere = 3u;
WF_HDI uint32_t hit_kind(uint32_t prim) { return prim >> 30; }
WF_HDI uint32_t hit_index(uint32_t prim) { return prim & 0x3fffffffu; }
WF_HDI uint32_t make_prim(uint32_t kind, uint32_t index) { return (kind << 30) | index; }

// The scene as kernels see it (passed by value, like the reference's Scene,
// include/scene/scene.cuh:117-161).
struct DeviceScene {
    const float4* triangles;
    const float4* normals;  // 3 float4 per triangle, or null
    const BvhNode* nodes;
    const Blas* blases;
    const Instance* instances;
    const uint32_t* mesh_linear;  // per BLAS, triangle positions in original order
    const uint32_t* tlas_leaves;  // (is_sphere << 31) | index
    const float4* spheres;
    const uint32_t* sphere_materials;
    const uint32_t* direct_spheres;
    const uint32_t* direct_instances;
    const Material* materials;
    const Light* lights;
    const Punctual* punctual;
    Environment env;
    BvhRef tlas;
    BvhRef direct_bvh;  // direct-list triangle BVH (root kNoRoot = linear scan)
    uint32_t static_first, static_count;
    uint32_t direct_first, direct_count;
    uint32_t direct_sphere_count;
    uint32_t direct_instance_count;
    uint32_t instance_count;
    uint32_t material_count;
    uint32_t light_count;
    uint32_t punctual_count;
    uint32_t directional_count;
    uint32_t any_alpha_reject;
    uint32_t black_background;
    uint32_t ignore_direct_light_occlusion;
    // textured materials (the shading stage and alpha-textured hits only)
    const MaterialTextures* material_textures;  // one per material, or null
    const uchar4* texels;                       // all textures, RGBA8
    const uint4* textures;                      // width, height, first texel
    const TriAttr* tri_attr;                    // per packed triangle, or null
    uint32_t texture_count;
    uint32_t use_normal_maps;
    float normal_map_min_cosine;
};

// ----------------------------------------------------------- parameters
struct Camera {
    V3 position, forward, right, up;
    float aspect_ratio;
    float tan_half_fov;  // tanf(verticalFov * 0.5f), camera.cuh:19
};

// Caustic gather requests of one bounce (filled in by the gather kernel): the
// term slot, the shading point and the two factors of
// throughput * (albedo * caustic).
struct GatherQueue {
    float4* position;    // xyz, global term index
    float4* normal;      // xyz, 1 = indirect (depth > 0)
    float4* throughput;  // xyz
    float4* albedo;      // xyz
    uint32_t* count;
    uint32_t capacity;
    uint32_t* dense;       // requests with many candidate photons (indices into the queue)
    uint32_t* dense_count;
};

struct PhotonGridView {
    const float4* position;   // sorted by cell; .w unused
    const float4* direction;
    const float4* flux;
    const uint32_t* cell_start;
    const uint32_t* cell_count;
    uint32_t resolution;
    V3 minimum, maximum;
    uint32_t enabled;  // grid present and gather on
};

struct RenderParams {
    uint32_t width, height;
    uint32_t max_depth, rr_start;
    uint32_t rng;
    uint32_t debug;
    float clamp;
    float gather_radius;
    Camera camera;
    PhotonGridView photons;
};

}  // namespace wf
