// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into or called by the
// product.  Only tests/ load the libraries this file is part of.
//
// The reference's asset path as a checker for the product's loaders: its
// OBJ and glTF loaders (src/scene/obj_loader.cpp, src/scene/gltf_loader.cpp,
// compiled with tinyobjloader, tinygltf and stb_image from the reference's
// extern/ tree by oracle/Makefile) and its scene assembly
// (src/scene/scene_host.cpp: assembleGltfScene, assembleCornellScene,
// assembleObjScene) build a HostScene, which is exported here in the C-ABI
// layouts of include/wavefront.h so a test can compare it field by field with
// the scene the product's loaders build; wfref_host_scene_upload turns it
// into a renderable reference scene.
#include "scene/environment.hpp"
#include "scene/gltf_loader.hpp"
#include "scene/obj_loader.hpp"
#include "scene/scene_host.hpp"

#include "../include/wavefront.h"

#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>

namespace {

struct HostSceneHandle {
    HostScene scene;
};

void put3(float* out, const Vec3& v) {
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

void put2(float* out, const Vec2& v) {
    out[0] = v.x;
    out[1] = v.y;
}

wf_texture_binding binding(const TextureBinding& b) {
    wf_texture_binding r;
    std::memset(&r, 0, sizeof(r));
    r.texture = b.texture;
    r.texcoord = b.texCoord;
    put2(r.offset, b.offset);
    put2(r.scale, b.scale);
    r.rotation = b.rotation;
    r.has_transform = b.hasTransform ? 1u : 0u;
    return r;
}

void triangle(const Triangle& t, wf_triangle& o, wf_triangle_attributes* a) {
    std::memset(&o, 0, sizeof(o));
    put3(o.v0, t.v0); put3(o.v1, t.v1); put3(o.v2, t.v2);
    put3(o.n0, t.n0); put3(o.n1, t.n1); put3(o.n2, t.n2);
    o.material = t.material;
    o.has_vertex_normals = t.hasVertexNormals ? 1u : 0u;
    if (!a) return;
    std::memset(a, 0, sizeof(*a));
    put2(a->uv[0], t.uv0); put2(a->uv[1], t.uv1); put2(a->uv[2], t.uv2);
    put2(a->uv1[0], t.uv1_0); put2(a->uv1[1], t.uv1_1); put2(a->uv1[2], t.uv1_2);
    put3(a->tangent, t.tangent); put3(a->bitangent, t.bitangent);
    put3(a->tangent1, t.tangent1); put3(a->bitangent1, t.bitangent1);
    put3(a->vertex_tangent[0], t.vertexTangent0);
    put3(a->vertex_tangent[1], t.vertexTangent1);
    put3(a->vertex_tangent[2], t.vertexTangent2);
    a->vertex_tangent_sign[0] = t.vertexTangentSign0;
    a->vertex_tangent_sign[1] = t.vertexTangentSign1;
    a->vertex_tangent_sign[2] = t.vertexTangentSign2;
    a->has_vertex_tangents = t.hasVertexTangents ? 1u : 0u;
    a->has_texcoords = t.hasTexcoords ? 1u : 0u;
    a->has_texcoords1 = t.hasTexcoords1 ? 1u : 0u;
}

const std::vector<Triangle>* triangle_list(const HostScene& h, int which, uint32_t mesh) {
    if (which == 0) return &h.triangles;
    if (which == 1) return &h.staticTriangles;
    if (which == 2 && mesh < h.meshes.size()) return &h.meshes[mesh].triangles;
    return nullptr;
}

}  // namespace

extern "C" {

// The reference's loadEnvironmentMap (src/scene/environment.cpp:66-82) on a
// Radiance .hdr file: *width and *height always, and with rgba non-null the
// width*height float4 texels.  Returns 0, or 1 when the reference throws.
int wfref_load_environment(const char* path, uint32_t* width, uint32_t* height, float* rgba) {
    try {
        HostEnvironment map = loadEnvironmentMap(path);
        *width = map.width;
        *height = map.height;
        if (rgba) std::memcpy(rgba, map.pixels.data(), sizeof(float) * 4 * map.pixels.size());
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfref_load_environment: %s\n", e.what());
        return 1;
    }
}

// The reference's preset assembly.  kind 0: assembleGltfScene(filename,
// scale, add_top_light) (the sponza preset); kind 1:
// assembleCornellScene(CornellSceneOptions) (cornell, hurricane, prism,
// crystal); kind 2: assembleObjScene(ObjSceneOptions) (deer); kind 3:
// assembleDemoScene(); kind 4: assembleRtWeekScene(filename).  NULL when the
// reference throws.
void* wfref_host_preset(int kind, const char* filename, float scale, const float* translation, int object_source,
                        int neutral_room, int remove_backdrop, int dielectric, int material_override,
                        int light_profile, int add_top_light, int acceleration) {
    try {
        auto handle = std::make_unique<HostSceneHandle>();
        Vec3 t(translation[0], translation[1], translation[2]);
        if (kind == 0) {
            handle->scene = assembleGltfScene(filename, scale, add_top_light != 0);
        } else if (kind == 1) {
            CornellSceneOptions o;
            o.filename = filename && filename[0] ? filename : nullptr;
            o.objectSource = CornellObjectSource(object_source);
            o.objectScale = scale;
            o.objectTranslation = t;
            o.neutralRoom = neutral_room != 0;
            o.removeBackdrop = remove_backdrop != 0;
            o.convertObjectMaterialsToDielectric = dielectric != 0;
            o.objectMaterialOverride = material_override;
            o.lightProfile = CornellLightProfile(light_profile);
            handle->scene = assembleCornellScene(o);
        } else if (kind == 3) {
            handle->scene = assembleDemoScene();
        } else if (kind == 4) {
            handle->scene = assembleRtWeekScene(filename);
        } else if (kind == 2) {
            ObjSceneOptions o;
            o.filename = filename;
            o.objectScale = scale;
            o.objectTranslation = t;
            o.acceleration = ObjAccelerationPolicy(acceleration);
            handle->scene = assembleObjScene(o);
        } else {
            return nullptr;
        }
        return handle.release();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "wfref_host_preset: %s\n", e.what());
        return nullptr;
    }
}

void wfref_host_scene_destroy(void* h) { delete static_cast<HostSceneHandle*>(h); }

HostScene* wfref_host_scene_get(void* h) { return &static_cast<HostSceneHandle*>(h)->scene; }

// counts: spheres, triangles, static triangles, meshes, instances,
// materials, textures, punctual lights, triangle lights, black background
void wfref_host_scene_counts(void* handle, uint64_t* counts) {
    const HostScene& h = static_cast<HostSceneHandle*>(handle)->scene;
    counts[0] = h.spheres.size();
    counts[1] = h.triangles.size();
    counts[2] = h.staticTriangles.size();
    counts[3] = h.meshes.size();
    counts[4] = h.instances.size();
    counts[5] = h.materials.size();
    counts[6] = h.textures.size();
    counts[7] = h.punctualLights.size();
    counts[8] = h.lights.size();
    counts[9] = h.blackBackground ? 1u : 0u;
}

uint64_t wfref_host_scene_triangle_count(void* handle, int which, uint32_t mesh) {
    const auto* list = triangle_list(static_cast<HostSceneHandle*>(handle)->scene, which, mesh);
    return list ? list->size() : 0;
}

// which 0: triangles, 1: static triangles, 2: mesh `mesh`
void wfref_host_scene_triangles(void* handle, int which, uint32_t mesh, wf_triangle* out,
                                wf_triangle_attributes* attributes) {
    const auto* list = triangle_list(static_cast<HostSceneHandle*>(handle)->scene, which, mesh);
    if (!list) return;
    for (size_t i = 0; i < list->size(); ++i) triangle((*list)[i], out[i], attributes ? &attributes[i] : nullptr);
}

void wfref_host_scene_materials(void* handle, wf_material* out, wf_material_textures* textures) {
    const HostScene& h = static_cast<HostSceneHandle*>(handle)->scene;
    for (size_t i = 0; i < h.materials.size(); ++i) {
        const Material& m = h.materials[i];
        wf_material& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.type = uint32_t(m.type);
        put3(o.albedo, m.albedo);
        put3(o.emission, m.emission);
        o.roughness = m.roughness;
        o.ior = m.ior;
        o.dispersion = m.dispersion;
        o.metallic = m.metallic;
        put3(o.attenuation_color, m.attenuationColor);
        o.attenuation_distance = m.attenuationDistance;
        o.volume_density = m.volumeDensity;
        o.opacity = m.opacity;
        o.alpha_cutoff = m.alphaCutoff;
        o.alpha_masked = m.alphaMasked ? 1u : 0u;
        o.specgloss_workflow = m.specularGlossinessWorkflow ? 1u : 0u;
        o.gltf_pbr = m.gltfPbrWorkflow ? 1u : 0u;
        put3(o.specular, m.specular);
        o.glossiness = m.glossiness;
        o.specular_weight = m.specularWeight;
        put3(o.specular_color, m.specularColor);
        o.clearcoat = m.clearcoat;
        o.clearcoat_roughness = m.clearcoatRoughness;
        if (!textures) continue;
        wf_material_textures& t = textures[i];
        t.normal_scale = m.normalScale;
        t.clearcoat_normal_scale = m.clearcoatNormalScale;
        t.albedo = binding(m.albedoTexture);
        t.metallic_roughness = binding(m.metallicRoughnessTexture);
        t.emissive = binding(m.emissiveTexture);
        t.normal = binding(m.normalTexture);
        t.thickness = binding(m.thicknessTexture);
        t.specular_glossiness = binding(m.specularGlossinessTexture);
        t.specular_weight = binding(m.specularWeightTexture);
        t.specular_color = binding(m.specularColorTexture);
        t.clearcoat = binding(m.clearcoatTexture);
        t.clearcoat_roughness = binding(m.clearcoatRoughnessTexture);
        t.clearcoat_normal = binding(m.clearcoatNormalTexture);
    }
}

void wfref_host_scene_instances(void* handle, wf_instance* out) {
    const HostScene& h = static_cast<HostSceneHandle*>(handle)->scene;
    for (size_t i = 0; i < h.instances.size(); ++i) {
        const SceneInstance& s = h.instances[i];
        wf_instance& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.mesh = s.meshIndex;
        o.material_override = s.materialOverride;
        o.accel = s.acceleration == AccelerationMode::Direct ? WF_ACCEL_DIRECT : WF_ACCEL_BVH;
        put3(o.local_to_world[0], s.transform.localToWorldX);
        put3(o.local_to_world[1], s.transform.localToWorldY);
        put3(o.local_to_world[2], s.transform.localToWorldZ);
        put3(o.world_to_local[0], s.transform.worldToLocalX);
        put3(o.world_to_local[1], s.transform.worldToLocalY);
        put3(o.world_to_local[2], s.transform.worldToLocalZ);
        put3(o.translation, s.transform.translation);
    }
}

void wfref_host_scene_spheres(void* handle, wf_sphere* out) {
    const HostScene& h = static_cast<HostSceneHandle*>(handle)->scene;
    for (size_t i = 0; i < h.spheres.size(); ++i) {
        const SceneSphere& s = h.spheres[i];
        std::memset(&out[i], 0, sizeof(out[i]));
        put3(out[i].center, s.geometry.center);
        out[i].radius = s.geometry.radius;
        out[i].material = s.geometry.material;
        out[i].accel = s.acceleration == AccelerationMode::Direct ? WF_ACCEL_DIRECT : WF_ACCEL_BVH;
    }
}

void wfref_host_scene_punctual(void* handle, wf_punctual_light* out) {
    const HostScene& h = static_cast<HostSceneHandle*>(handle)->scene;
    for (size_t i = 0; i < h.punctualLights.size(); ++i) {
        const PunctualLight& l = h.punctualLights[i];
        std::memset(&out[i], 0, sizeof(out[i]));
        out[i].type = uint32_t(l.type);
        put3(out[i].position, l.position);
        put3(out[i].direction, l.direction);
        put3(out[i].intensity, l.intensity);
        out[i].range = l.range;
        out[i].inner_cone_cos = l.innerConeCos;
        out[i].outer_cone_cos = l.outerConeCos;
    }
}

// width and height of texture i; its RGBA8 texels into rgba when not NULL
void wfref_host_scene_texture(void* handle, uint32_t i, uint32_t* size, uint8_t* rgba) {
    const HostScene& h = static_cast<HostSceneHandle*>(handle)->scene;
    const ObjTexture& t = h.textures.at(i);
    size[0] = t.width;
    size[1] = t.height;
    if (rgba) std::memcpy(rgba, t.pixels.data(), t.pixels.size());
}

}  // extern "C"
