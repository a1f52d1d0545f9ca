// Host scene build: restates the reference's upload path
// (src/scene/scene.cu:82-294,336-389), its scene-assembly light registration
// (src/scene/scene_host.cpp:60-106) and its environment distribution
// (src/scene/environment.cpp:10-64), producing the packed device layout of
// wf_device.cuh.  Floating-point expressions keep the reference's order so the
// light and environment tables are bit-identical to the reference's.
#include "wf_internal.h"
#include "wf_bvh_gpu.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>

namespace wf {

// Smallest BVH2 input the GPU builder takes; smaller trees build on the host
// in well under a millisecond.
constexpr uint32_t kGpuBvhMinPrimitives = 4096;

namespace {
thread_local std::string g_error;

uint32_t float_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
float bits_float(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
V3 vec(const float* p) { return V3{p[0], p[1], p[2]}; }

// transformVector(T, v) + T.translation, include/scene/scene.cuh:39-42.
V3 to_world(const wf_instance& in, V3 v) {
    V3 x = vec(in.local_to_world[0]), y = vec(in.local_to_world[1]), z = vec(in.local_to_world[2]);
    return x * v.x + y * v.y + z * v.z + vec(in.translation);
}

BvhBox triangle_box(const wf_triangle& t) {
    BvhBox b;
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(std::min(t.v0[a], t.v1[a]), t.v2[a]);
        b.hi[a] = std::max(std::max(t.v0[a], t.v1[a]), t.v2[a]);
    }
    return b;
}

void grow(Box& b, const BvhBox& o) {
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(b.lo[a], o.lo[a]);
        b.hi[a] = std::max(b.hi[a], o.hi[a]);
    }
}

Box to_box(const BvhBox& b) {
    Box r;
    for (int a = 0; a < 3; ++a) { r.lo[a] = b.lo[a]; r.hi[a] = b.hi[a]; }
    return r;
}

// Converts a binary tree (bvh_build.h) to 64-byte child-box nodes in DFS
// pre-order.  `leaf_ref(prim)` returns the packed position of a primitive;
// for triangle BVHs `on_leaf` is called in DFS order to assign positions.
struct Converter {
    const std::vector<BvhBinaryNode>& bin;
    std::vector<BvhNode>& out;
    std::function<uint32_t(uint32_t)> leaf_ref;

    int child_ref(uint32_t b) {
        const BvhBinaryNode& n = bin[b];
        if (n.left == kInvalidChild) return ~int(leaf_ref(n.right));
        return convert(b);
    }
    int convert(uint32_t b) {
        const BvhBinaryNode& n = bin[b];
        int index = int(out.size());
        out.push_back(BvhNode{});
        const BvhBox& l = bin[n.left].box;
        const BvhBox& r = bin[n.right].box;
        int lref = child_ref(n.left);
        int rref = child_ref(n.right);
        BvhNode& node = out[size_t(index)];
        node.lxy = make_float4(l.lo[0], l.hi[0], l.lo[1], l.hi[1]);
        node.rxy = make_float4(r.lo[0], r.hi[0], r.lo[1], r.hi[1]);
        node.lrz = make_float4(l.lo[2], l.hi[2], r.lo[2], r.hi[2]);
        node.child = make_int4(lref, rref, 0, 0);
        return index;
    }
    BvhRef root() {
        BvhRef ref{kNoRoot, {}};
        if (bin.empty()) return ref;
        uint32_t r = uint32_t(bin.size() - 1);
        ref.box = to_box(bin[r].box);
        ref.root = child_ref(r);
        return ref;
    }
};

// DFS leaf order of a binary tree (left first): the packing order of a BLAS.
void leaf_order(const std::vector<BvhBinaryNode>& bin, std::vector<uint32_t>& order) {
    order.clear();
    if (bin.empty()) return;
    std::vector<uint32_t> stack{uint32_t(bin.size() - 1)};
    while (!stack.empty()) {
        uint32_t b = stack.back();
        stack.pop_back();
        const BvhBinaryNode& n = bin[b];
        if (n.left == kInvalidChild) {
            order.push_back(n.right);
            continue;
        }
        stack.push_back(n.right);
        stack.push_back(n.left);
    }
}

// `attr`: the triangle's texture coordinates and tangents, or null (zeros);
// stored only when the scene carries attributes at all.
void pack_triangle(HostScene& s, const wf_triangle& t, uint32_t original, uint32_t light, bool with_normals,
                   const wf_triangle_attributes* attr, bool with_attributes) {
    if (with_attributes) {
        TriAttr a{};
        static_assert(sizeof(wf_triangle_attributes) <= sizeof(TriAttr), "attribute record fits");
        if (attr) std::memcpy(&a, attr, sizeof(wf_triangle_attributes));
        s.tri_attr.push_back(a);
    }
    uint32_t flags = original | (t.has_vertex_normals ? kTriHasNormals : 0u);
    s.triangles.push_back(make_float4(t.v0[0], t.v0[1], t.v0[2], bits_float(flags)));
    s.triangles.push_back(make_float4(t.v1[0], t.v1[1], t.v1[2], bits_float(t.material)));
    s.triangles.push_back(make_float4(t.v2[0], t.v2[1], t.v2[2], bits_float(light)));
    if (with_normals) {
        s.normals.push_back(make_float4(t.n0[0], t.n0[1], t.n0[2], 0.0f));
        s.normals.push_back(make_float4(t.n1[0], t.n1[1], t.n1[2], 0.0f));
        s.normals.push_back(make_float4(t.n2[0], t.n2[1], t.n2[2], 0.0f));
    }
}

Material to_material(const wf_material& m) {
    Material r{};
    r.type = m.type;
    r.flags = (m.gltf_pbr ? kMatGltfPbr : 0u) | (m.specgloss_workflow ? kMatSpecGlossWorkflow : 0u) |
              (m.alpha_masked && m.opacity < m.alpha_cutoff ? kMatAlphaReject : 0u);
    r.roughness = m.roughness;
    r.ior = m.ior;
    r.albedo = vec(m.albedo);
    r.emission = vec(m.emission);
    r.metallic = m.metallic;
    r.dispersion = m.dispersion;
    r.attenuation_color = vec(m.attenuation_color);
    r.attenuation_distance = m.attenuation_distance;
    r.volume_density = m.volume_density;
    r.glossiness = m.glossiness;
    r.specular = vec(m.specular);
    r.specular_weight = m.specular_weight;
    r.specular_color = vec(m.specular_color);
    r.clearcoat = m.clearcoat;
    r.clearcoat_roughness = m.clearcoat_roughness;
    return r;
}

struct PendingLight {
    Light light;
    float weight;
};

// One registered triangle light (scene_host.cpp:66-73 and 94-104).
PendingLight make_light(V3 v0, V3 v1, V3 v2, uint32_t material, const wf_material& m) {
    V3 normal = normalize(cross(v1 - v0, v2 - v0));
    float area = 0.5f * length(cross(v1 - v0, v2 - v0));
    float power = area * (0.2126f * m.emission[0] + 0.7152f * m.emission[1] + 0.0722f * m.emission[2]);
    PendingLight p{};
    p.light.v0 = v0;
    p.light.v1 = v1;
    p.light.v2 = v2;
    p.light.normal = normal;
    p.light.area = area;
    p.light.material = material;
    p.light.selection_pdf = 0.0f;
    p.weight = power;
    return p;
}

// uploadTriangleLights, src/scene/scene.cu:82-121 (Vose alias in float).
void finish_lights(std::vector<PendingLight>& pending, std::vector<Light>& lights) {
    lights.clear();
    if (pending.empty()) return;
    float total = 0.0f;
    for (const PendingLight& p : pending) total += p.weight;
    size_t n = pending.size();
    std::vector<float> scaled(n);
    std::vector<uint32_t> small, large;
    for (uint32_t i = 0; i < n; ++i) {
        pending[i].light.selection_pdf = pending[i].weight / total;
        scaled[i] = pending[i].light.selection_pdf * n;
        (scaled[i] < 1.0f ? small : large).push_back(i);
    }
    std::vector<float> alias_probability(n);
    std::vector<uint32_t> alias(n);
    while (!small.empty() && !large.empty()) {
        uint32_t low = small.back();
        small.pop_back();
        uint32_t high = large.back();
        large.pop_back();
        alias_probability[low] = scaled[low];
        alias[low] = high;
        scaled[high] = scaled[high] + scaled[low] - 1.0f;
        (scaled[high] < 1.0f ? small : large).push_back(high);
    }
    for (uint32_t i : small) { alias_probability[i] = 1.0f; alias[i] = i; }
    for (uint32_t i : large) { alias_probability[i] = 1.0f; alias[i] = i; }
    lights.resize(n);
    for (size_t i = 0; i < n; ++i) {
        lights[i] = pending[i].light;
        lights[i].alias_probability = alias_probability[i];
        lights[i].alias = alias[i];
    }
}

}  // namespace

wf_status fail(wf_status status, const char* format, ...) {
    char buffer[512];
    va_list args;
    va_start(args, format);
    std::vsnprintf(buffer, sizeof(buffer), format, args);
    va_end(args);
    g_error = buffer;
    return status;
}

const char* last_error_text() { return g_error.c_str(); }

wf_status build_host_scene(const wf_scene_desc* d, HostScene& s) {
    if (!d) return fail(WF_ERR_INVALID_ARG, "scene description is null");
    auto need = [](const void* p, uint32_t n) { return n == 0 || p != nullptr; };
    if (!need(d->spheres, d->sphere_count) || !need(d->triangles, d->triangle_count) ||
        !need(d->static_triangles, d->static_triangle_count) || !need(d->meshes, d->mesh_count) ||
        !need(d->instances, d->instance_count) || !need(d->materials, d->material_count) ||
        !need(d->punctual_lights, d->punctual_light_count))
        return fail(WF_ERR_INVALID_ARG, "scene description has a null array with a nonzero count");
    uint32_t nm = d->material_count;
    auto bad_material = [nm](uint32_t m) { return m >= nm; };
    for (uint32_t i = 0; i < d->sphere_count; ++i)
        if (bad_material(d->spheres[i].material)) return fail(WF_ERR_INVALID_ARG, "sphere %u material out of range", i);
    auto check_tris = [&](const wf_triangle* t, uint32_t n, const char* what) -> wf_status {
        for (uint32_t i = 0; i < n; ++i)
            if (bad_material(t[i].material)) return fail(WF_ERR_INVALID_ARG, "%s %u material out of range", what, i);
        return WF_OK;
    };
    if (wf_status e = check_tris(d->triangles, d->triangle_count, "triangle")) return e;
    if (wf_status e = check_tris(d->static_triangles, d->static_triangle_count, "static triangle")) return e;
    uint64_t total_triangles = uint64_t(d->triangle_count) + d->static_triangle_count;
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        if (!need(d->meshes[m].triangles, d->meshes[m].triangle_count))
            return fail(WF_ERR_INVALID_ARG, "mesh %u has null triangles", m);
        if (wf_status e = check_tris(d->meshes[m].triangles, d->meshes[m].triangle_count, "mesh triangle")) return e;
        total_triangles += d->meshes[m].triangle_count;
    }
    if (total_triangles >= (1ull << 30)) return fail(WF_ERR_CAPACITY, "more than 2^30 triangles");
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const wf_instance& in = d->instances[i];
        if (in.mesh >= d->mesh_count) return fail(WF_ERR_INVALID_ARG, "instance %u mesh out of range", i);
        if (in.material_override != WF_NO_MATERIAL && bad_material(in.material_override))
            return fail(WF_ERR_INVALID_ARG, "instance %u material override out of range", i);
    }
    for (uint32_t i = 0; i < d->punctual_light_count; ++i)
        if (d->punctual_lights[i].type > WF_LIGHT_DIRECTIONAL)
            return fail(WF_ERR_INVALID_ARG, "punctual light %u has an unknown type", i);

    s = HostScene{};
    // --- textures (uploadTextures, scene.cu:44-80): one RGBA8 texel pool
    for (uint32_t i = 0; i < d->texture_count; ++i) {
        const wf_texture& t = d->textures[i];
        if (t.width == 0 || t.height == 0 || !t.rgba)
            return fail(WF_ERR_INVALID_ARG, "texture %u is empty or has no texels", i);
        s.textures.push_back(make_uint4(t.width, t.height, uint32_t(s.texels.size()), 0u));
        size_t count = size_t(t.width) * t.height;
        if (s.texels.size() + count > 0xffffffffull) return fail(WF_ERR_CAPACITY, "more than 2^32 texels");
        const uchar4* p = reinterpret_cast<const uchar4*>(t.rgba);
        s.texels.insert(s.texels.end(), p, p + count);
    }
    for (uint32_t i = 0; i < nm; ++i) {
        s.materials.push_back(to_material(d->materials[i]));
        if (d->materials[i].type > WF_MAT_SPECGLOSS) return fail(WF_ERR_INVALID_ARG, "material %u has an unknown type", i);
        if (d->material_textures) {
            // sampleTexture ignores bindings past textureCount
            // (device_traversal.cuh:342-343): they do not flag the material.
            const wf_material_textures& w = d->material_textures[i];
            MaterialTextures mt{};
            mt.normal_scale = w.normal_scale;
            mt.clearcoat_normal_scale = w.clearcoat_normal_scale;
            mt.opacity = d->materials[i].opacity;
            mt.alpha_cutoff = d->materials[i].alpha_cutoff;
            const wf_texture_binding* slots[kTexSlots] = {
                &w.albedo, &w.metallic_roughness, &w.emissive, &w.normal, &w.thickness, &w.specular_glossiness,
                &w.specular_weight, &w.specular_color, &w.clearcoat, &w.clearcoat_roughness, &w.clearcoat_normal};
            bool any = false;
            for (uint32_t k = 0; k < kTexSlots; ++k) {
                const wf_texture_binding& b = *slots[k];
                mt.slot[k] = TexBinding{b.texture, b.texcoord, b.offset[0], b.offset[1], b.scale[0], b.scale[1],
                                        b.rotation, b.has_transform};
                any = any || b.texture < d->texture_count;
            }
            Material& m = s.materials.back();
            if (any) {
                m.flags |= kMatTextured;
                s.textured = true;
            }
            if (d->materials[i].alpha_masked && w.albedo.texture < d->texture_count) {
                m.flags = (m.flags & ~kMatAlphaReject) | kMatAlphaTexture;  // opacity * albedo.a per hit
                s.alpha_textures = true;
            }
            s.material_textures.push_back(mt);
        }
        if (s.materials.back().flags & (kMatAlphaReject | kMatAlphaTexture)) s.any_alpha_reject = true;
    }
    s.use_normal_maps = d->disable_normal_maps == 0;
    s.normal_map_min_cosine = d->normal_map_minimum_cosine;
    bool with_attributes = d->triangle_attributes != nullptr || d->static_triangle_attributes != nullptr;
    for (uint32_t m = 0; m < d->mesh_count; ++m) with_attributes = with_attributes || d->meshes[m].attributes;
    bool with_normals = false;
    auto scan_normals = [&](const wf_triangle* t, uint32_t n) {
        for (uint32_t i = 0; i < n && !with_normals; ++i) with_normals = t[i].has_vertex_normals != 0;
    };
    scan_normals(d->triangles, d->triangle_count);
    scan_normals(d->static_triangles, d->static_triangle_count);
    for (uint32_t m = 0; m < d->mesh_count; ++m) scan_normals(d->meshes[m].triangles, d->meshes[m].triangle_count);

    auto is_emissive = [&](uint32_t material) { return d->materials[material].type == WF_MAT_EMISSIVE; };
    bool register_lights = d->register_triangle_lights != 0;

    // --- light registration: addMeshTriangleLights then addStaticTriangleLights.
    std::vector<std::vector<uint32_t>> mesh_light(d->mesh_count);
    std::vector<uint32_t> mesh_light_count(d->mesh_count, 0);
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        mesh_light[m].assign(d->meshes[m].triangle_count, kInvalid);
        if (!register_lights) continue;
        uint32_t local = 0;
        for (uint32_t i = 0; i < d->meshes[m].triangle_count; ++i)
            if (is_emissive(d->meshes[m].triangles[i].material)) mesh_light[m][i] = local++;
        mesh_light_count[m] = local;
    }
    std::vector<PendingLight> pending;
    if (register_lights) {
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            const wf_instance& in = d->instances[i];
            const wf_mesh& mesh = d->meshes[in.mesh];
            for (uint32_t k = 0; k < mesh.triangle_count; ++k) {
                if (mesh_light[in.mesh][k] == kInvalid) continue;
                const wf_triangle& t = mesh.triangles[k];
                V3 v0 = to_world(in, vec(t.v0)), v1 = to_world(in, vec(t.v1)), v2 = to_world(in, vec(t.v2));
                pending.push_back(make_light(v0, v1, v2, t.material, d->materials[t.material]));
            }
        }
    }
    std::vector<uint32_t> static_light(d->static_triangle_count, kInvalid);
    if (register_lights) {
        for (uint32_t i = 0; i < d->static_triangle_count; ++i) {
            const wf_triangle& t = d->static_triangles[i];
            if (!is_emissive(t.material)) continue;
            static_light[i] = uint32_t(pending.size());
            pending.push_back(make_light(vec(t.v0), vec(t.v1), vec(t.v2), t.material, d->materials[t.material]));
        }
    }
    finish_lights(pending, s.lights);

    for (int a = 0; a < 3; ++a) { s.bounds.lo[a] = INFINITY; s.bounds.hi[a] = -INFINITY; }

    // --- meshes / BLAS (uploadMeshInstances, scene.cu:123-173)
    std::vector<bool> needs_bvh(d->mesh_count, false);
    for (uint32_t i = 0; i < d->instance_count; ++i)
        if (d->instances[i].accel == WF_ACCEL_BVH) needs_bvh[d->instances[i].mesh] = true;
    int threads = int(d->build_threads);
    // BVH2 builds: the host binned-SAH builder, or the GPU PLOC builder for
    // large inputs (falls back to the host builder on any failure or a tree
    // deeper than kMaxBvhDepth).
    auto build_bvh = [&](const BvhBox* prims, uint32_t n, std::vector<BvhBinaryNode>& out) {
        auto t0 = std::chrono::steady_clock::now();
        bool done = false;
        if (d->bvh_builder == WF_BVH_GPU_PLOC && n >= kGpuBvhMinPrimitives) {
            char why[256] = {0};
            done = build_binary_bvh_gpu(prims, n, out, kMaxBvhDepth, why, sizeof(why), threads);
            if (done) ++s.gpu_bvh_builds;
        }
        if (!done) build_binary_bvh(prims, n, out, threads);
        s.bvh_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    std::vector<BvhBox> boxes;
    std::vector<BvhBinaryNode> bin;
    std::vector<uint32_t> order;
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        const wf_mesh& mesh = d->meshes[m];
        Blas b{};
        b.bvh = BvhRef{kNoRoot, {}};
        b.first = uint32_t(s.triangles.size() / 3);
        b.count = mesh.triangle_count;
        b.first_linear = uint32_t(s.mesh_linear.size());
        s.mesh_linear.resize(s.mesh_linear.size() + mesh.triangle_count);
        if (needs_bvh[m] && mesh.triangle_count > 0) {
            boxes.resize(mesh.triangle_count);
            for (uint32_t i = 0; i < mesh.triangle_count; ++i) boxes[i] = triangle_box(mesh.triangles[i]);
            build_bvh(boxes.data(), mesh.triangle_count, bin);
            leaf_order(bin, order);
            std::vector<uint32_t> position(mesh.triangle_count);
            for (uint32_t k = 0; k < order.size(); ++k) {
                uint32_t prim = order[k];
                position[prim] = b.first + k;
                pack_triangle(s, mesh.triangles[prim], prim, mesh_light[m][prim], with_normals,
                              mesh.attributes ? &mesh.attributes[prim] : nullptr, with_attributes);
            }
            for (uint32_t i = 0; i < mesh.triangle_count; ++i) s.mesh_linear[b.first_linear + i] = position[i];
            Converter c{bin, s.nodes, [&](uint32_t prim) { return position[prim]; }};
            b.bvh = c.root();
        } else {
            for (uint32_t i = 0; i < mesh.triangle_count; ++i) {
                pack_triangle(s, mesh.triangles[i], i, mesh_light[m][i], with_normals,
                              mesh.attributes ? &mesh.attributes[i] : nullptr, with_attributes);
                s.mesh_linear[b.first_linear + i] = b.first + i;
            }
        }
        s.blases.push_back(b);
    }
    uint32_t light_offset = 0;
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const wf_instance& in = d->instances[i];
        Instance out{};
        out.w2l_x = make_float4(in.world_to_local[0][0], in.world_to_local[0][1], in.world_to_local[0][2], in.translation[0]);
        out.w2l_y = make_float4(in.world_to_local[1][0], in.world_to_local[1][1], in.world_to_local[1][2], in.translation[1]);
        out.w2l_z = make_float4(in.world_to_local[2][0], in.world_to_local[2][1], in.world_to_local[2][2], in.translation[2]);
        out.l2w_x = make_float4(in.local_to_world[0][0], in.local_to_world[0][1], in.local_to_world[0][2], 0.0f);
        out.l2w_y = make_float4(in.local_to_world[1][0], in.local_to_world[1][1], in.local_to_world[1][2], 0.0f);
        out.l2w_z = make_float4(in.local_to_world[2][0], in.local_to_world[2][1], in.local_to_world[2][2], 0.0f);
        out.blas = in.mesh;
        out.light_offset = light_offset;
        out.material_override = in.material_override;
        s.instances.push_back(out);
        light_offset += mesh_light_count[in.mesh];
    }

    // --- spheres + TLAS (uploadSceneTlas, scene.cu:175-239)
    std::vector<BvhBox> leaf_boxes;
    for (uint32_t i = 0; i < d->sphere_count; ++i) {
        const wf_sphere& sp = d->spheres[i];
        s.spheres.push_back(make_float4(sp.center[0], sp.center[1], sp.center[2], sp.radius));
        s.sphere_materials.push_back(sp.material);
        float r = fabsf(sp.radius);
        BvhBox b;
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = nextafterf(sp.center[a] - r, -INFINITY);
            b.hi[a] = nextafterf(sp.center[a] + r, INFINITY);
        }
        if (sp.accel == WF_ACCEL_DIRECT) {
            s.direct_spheres.push_back(i);
            if (r < 100.0f) grow(s.bounds, b);  // a ground sphere would swamp the bounds
            continue;
        }
        grow(s.bounds, b);
        leaf_boxes.push_back(b);
        s.tlas_leaves.push_back(0x80000000u | i);
    }
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const wf_instance& in = d->instances[i];
        if (in.accel == WF_ACCEL_DIRECT) {
            s.direct_instances.push_back(i);
            continue;
        }
        const Blas& blas = s.blases[in.mesh];
        if (d->meshes[in.mesh].triangle_count == 0) continue;
        const Box& lb = blas.bvh.box;
        BvhBox w;
        for (int a = 0; a < 3; ++a) { w.lo[a] = INFINITY; w.hi[a] = -INFINITY; }
        for (uint32_t corner = 0; corner < 8; ++corner) {
            V3 local{(corner & 1) ? lb.hi[0] : lb.lo[0], (corner & 2) ? lb.hi[1] : lb.lo[1],
                     (corner & 4) ? lb.hi[2] : lb.lo[2]};
            V3 x = vec(in.local_to_world[0]), y = vec(in.local_to_world[1]), z = vec(in.local_to_world[2]);
            V3 p = x * local.x + y * local.y + z * local.z + vec(in.translation);
            w.lo[0] = fminf(w.lo[0], p.x); w.lo[1] = fminf(w.lo[1], p.y); w.lo[2] = fminf(w.lo[2], p.z);
            w.hi[0] = fmaxf(w.hi[0], p.x); w.hi[1] = fmaxf(w.hi[1], p.y); w.hi[2] = fmaxf(w.hi[2], p.z);
        }
        grow(s.bounds, w);
        leaf_boxes.push_back(w);
        s.tlas_leaves.push_back(i);
    }
    if (!leaf_boxes.empty()) {
        build_bvh(leaf_boxes.data(), uint32_t(leaf_boxes.size()), bin);
        Converter c{bin, s.nodes, [](uint32_t leaf) { return leaf; }};
        s.tlas = c.root();
    }

    // --- static triangles (linear, original order)
    s.static_first = uint32_t(s.triangles.size() / 3);
    s.static_count = d->static_triangle_count;
    for (uint32_t i = 0; i < d->static_triangle_count; ++i) {
        pack_triangle(s, d->static_triangles[i], i, static_light[i], with_normals,
                      d->static_triangle_attributes ? &d->static_triangle_attributes[i] : nullptr, with_attributes);
        grow(s.bounds, triangle_box(d->static_triangles[i]));
    }

    // --- direct triangle list: own BVH only when the scene has no meshes
    // (uploadScene, scene.cu:361-375; otherwise intersectDirectTriangles scans).
    s.direct_first = uint32_t(s.triangles.size() / 3);
    s.direct_count = d->triangle_count;
    if (d->triangle_count > 0 && d->mesh_count == 0) {
        boxes.resize(d->triangle_count);
        for (uint32_t i = 0; i < d->triangle_count; ++i) boxes[i] = triangle_box(d->triangles[i]);
        build_bvh(boxes.data(), d->triangle_count, bin);
        leaf_order(bin, order);
        std::vector<uint32_t> position(d->triangle_count);
        for (uint32_t k = 0; k < order.size(); ++k) {
            position[order[k]] = s.direct_first + k;
            pack_triangle(s, d->triangles[order[k]], order[k], kInvalid, with_normals,
                          d->triangle_attributes ? &d->triangle_attributes[order[k]] : nullptr, with_attributes);
        }
        Converter c{bin, s.nodes, [&](uint32_t prim) { return position[prim]; }};
        s.direct_bvh = c.root();
    } else {
        for (uint32_t i = 0; i < d->triangle_count; ++i)
            pack_triangle(s, d->triangles[i], i, kInvalid, with_normals,
                          d->triangle_attributes ? &d->triangle_attributes[i] : nullptr, with_attributes);
    }
    for (uint32_t i = 0; i < d->triangle_count; ++i) grow(s.bounds, triangle_box(d->triangles[i]));

    // --- punctual lights: directional prefix (stable_partition, scene.cu:346-351)
    for (int pass = 0; pass < 2; ++pass)
        for (uint32_t i = 0; i < d->punctual_light_count; ++i) {
            const wf_punctual_light& l = d->punctual_lights[i];
            bool directional = l.type == WF_LIGHT_DIRECTIONAL;
            if (directional != (pass == 0)) continue;
            Punctual p{};
            p.type = l.type;
            p.position = vec(l.position);
            p.direction = vec(l.direction);
            p.intensity = vec(l.intensity);
            p.range = l.range;
            p.inner_cone_cos = l.inner_cone_cos;
            p.outer_cone_cos = l.outer_cone_cos;
            s.punctual.push_back(p);
            if (directional) ++s.directional_count;
        }
    s.black_background = d->black_background != 0;
    s.ignore_occlusion = d->ignore_direct_light_occlusion != 0;
    return WF_OK;
}

float environment_solid_angle(uint32_t row, uint32_t width, uint32_t height) {
    constexpr double pi = 3.14159265358979323846;
    return static_cast<float>((4.0 * pi / width) * wfm::sin(pi * (row + 0.5) / height) * wfm::sin(pi / (2.0 * height)));
}

wf_status build_environment(const wf_environment* env, HostEnvironment& map) {
    uint64_t count = uint64_t(env->width) * env->height;
    if (count == 0 || count > std::numeric_limits<uint32_t>::max() || !env->rgba)
        return fail(WF_ERR_INVALID_ARG, "invalid HDR environment dimensions");
    if (!std::isfinite(env->intensity) || env->intensity < 0 || !std::isfinite(env->rotation_degrees))
        return fail(WF_ERR_INVALID_ARG, "invalid HDR environment upload");
    map.width = env->width;
    map.height = env->height;
    map.pixels.resize(count);
    for (uint64_t i = 0; i < count; ++i) {
        const float* p = env->rgba + 4 * i;
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]) || p[0] < 0 || p[1] < 0 || p[2] < 0)
            return fail(WF_ERR_INVALID_ARG, "HDR environment contains negative or non-finite radiance");
        map.pixels[i] = make_float4(p[0], p[1], p[2], p[3]);
    }
    uint32_t w = map.width, h = map.height;
    std::vector<double> weights(count);
    double total = 0.0;
    constexpr double filter[3] = {0.125, 0.75, 0.125};
    for (uint32_t i = 0; i < count; ++i) {
        uint32_t x = i % w, y = i / w;
        uint32_t columns[3] = {x ? x - 1 : w - 1, x, x + 1 < w ? x + 1 : 0};
        uint32_t rows[3] = {y ? y - 1 : 0, y, y + 1 < h ? y + 1 : h - 1};
        double average = 0;
        for (int row = 0; row < 3; ++row)
            for (int col = 0; col < 3; ++col) {
                const float4& p = map.pixels[uint64_t(rows[row]) * w + columns[col]];
                average += filter[row] * filter[col] * (0.2126 * double(p.x) + 0.7152 * double(p.y) + 0.0722 * double(p.z));
            }
        weights[i] = average * environment_solid_angle(y, w, h);
        total += weights[i];
    }
    constexpr double four_pi = 12.5663706143591729538;
    map.probabilities.resize(count);
    map.alias.resize(count);
    double sum = 0;
    for (uint32_t i = 0; i < count; ++i) {
        double uniform = environment_solid_angle(i / w, w, h) / four_pi;
        map.probabilities[i] = static_cast<float>(total > 0 ? .99 * weights[i] / total + .01 * uniform : uniform);
        sum += map.probabilities[i];
    }
    std::vector<uint32_t> small, large;
    for (uint32_t i = 0; i < count; ++i) {
        map.probabilities[i] /= sum;
        weights[i] = double(map.probabilities[i]) * count;
        (weights[i] < 1.0 ? small : large).push_back(i);
    }
    while (!small.empty() && !large.empty()) {
        uint32_t low = small.back();
        small.pop_back();
        uint32_t high = large.back();
        large.pop_back();
        map.alias[low] = make_float2(static_cast<float>(weights[low]), bits_float(high));
        weights[high] += weights[low] - 1;
        (weights[high] < 1.0 ? small : large).push_back(high);
    }
    for (uint32_t i : small) map.alias[i] = make_float2(1.0f, bits_float(i));
    for (uint32_t i : large) map.alias[i] = make_float2(1.0f, bits_float(i));
    map.row_solid_angle.resize(h);
    for (uint32_t y = 0; y < h; ++y) map.row_solid_angle[y] = environment_solid_angle(y, w, h);
    map.intensity = env->intensity;
    map.rotation = std::fmod(env->rotation_degrees, 360.0f) * (3.14159265359f / 180.0f);
    return WF_OK;
}

}  // namespace wf
