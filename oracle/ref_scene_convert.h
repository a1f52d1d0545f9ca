// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// The C-ABI scene description (include/wavefront.h) as the reference's
// HostScene (include/scene/scene_host.hpp), for the two builds of the
// reference renderer in this directory: the host build (ref_harness.cpp) and
// the sm_100a build (ref_cuda_harness.cu).  Light registration runs the
// reference's own code (ref_scene_host_tu.cpp).
#pragma once

#include <cstdint>
#include <utility>

#include "scene/scene_host.hpp"

#include "../include/wavefront.h"

void wfref_register_lights(HostScene& scene);  // ref_scene_host_tu.cpp

namespace wfref {

inline Vec3 v3(const float* p) { return Vec3(p[0], p[1], p[2]); }

inline Vec2 v2(const float* p) { return Vec2{p[0], p[1]}; }

inline Triangle to_triangle(const wf_triangle& t, const wf_triangle_attributes* a = nullptr) {
    Triangle r{};
    r.v0 = v3(t.v0); r.v1 = v3(t.v1); r.v2 = v3(t.v2);
    r.n0 = v3(t.n0); r.n1 = v3(t.n1); r.n2 = v3(t.n2);
    r.material = t.material;
    r.lightIndex = invalidLightIndex;
    r.hasVertexNormals = t.has_vertex_normals != 0;
    if (a) {
        r.uv0 = v2(a->uv[0]); r.uv1 = v2(a->uv[1]); r.uv2 = v2(a->uv[2]);
        r.uv1_0 = v2(a->uv1[0]); r.uv1_1 = v2(a->uv1[1]); r.uv1_2 = v2(a->uv1[2]);
        r.tangent = v3(a->tangent); r.bitangent = v3(a->bitangent);
        r.tangent1 = v3(a->tangent1); r.bitangent1 = v3(a->bitangent1);
        r.vertexTangent0 = v3(a->vertex_tangent[0]);
        r.vertexTangent1 = v3(a->vertex_tangent[1]);
        r.vertexTangent2 = v3(a->vertex_tangent[2]);
        r.vertexTangentSign0 = a->vertex_tangent_sign[0];
        r.vertexTangentSign1 = a->vertex_tangent_sign[1];
        r.vertexTangentSign2 = a->vertex_tangent_sign[2];
        r.hasVertexTangents = a->has_vertex_tangents != 0;
        r.hasTexcoords = a->has_texcoords != 0;
        r.hasTexcoords1 = a->has_texcoords1 != 0;
    }
    return r;
}

inline TextureBinding to_binding(const wf_texture_binding& b) {
    TextureBinding r;
    r.texture = b.texture;
    r.texCoord = b.texcoord;
    r.offset = Vec2{b.offset[0], b.offset[1]};
    r.scale = Vec2{b.scale[0], b.scale[1]};
    r.rotation = b.rotation;
    r.hasTransform = b.has_transform != 0;
    return r;
}

inline void apply_textures(Material& r, const wf_material_textures& t) {
    r.normalScale = t.normal_scale;
    r.clearcoatNormalScale = t.clearcoat_normal_scale;
    r.albedoTexture = to_binding(t.albedo);
    r.metallicRoughnessTexture = to_binding(t.metallic_roughness);
    r.emissiveTexture = to_binding(t.emissive);
    r.normalTexture = to_binding(t.normal);
    r.thicknessTexture = to_binding(t.thickness);
    r.specularGlossinessTexture = to_binding(t.specular_glossiness);
    r.specularWeightTexture = to_binding(t.specular_weight);
    r.specularColorTexture = to_binding(t.specular_color);
    r.clearcoatTexture = to_binding(t.clearcoat);
    r.clearcoatRoughnessTexture = to_binding(t.clearcoat_roughness);
    r.clearcoatNormalTexture = to_binding(t.clearcoat_normal);
}

// Scene::useNormalMaps / normalMapMinimumCosine (include/scene/scene.cuh:159-160).
inline void apply_normal_map_settings(Scene& scene, const wf_scene_desc* d) {
    scene.useNormalMaps = d->disable_normal_maps == 0;
    scene.normalMapMinimumCosine = d->normal_map_minimum_cosine;
}

inline Material to_material(const wf_material& m) {
    Material r{};
    r.type = MaterialType(m.type);
    r.albedo = v3(m.albedo);
    r.emission = v3(m.emission);
    r.roughness = m.roughness;
    r.ior = m.ior;
    r.dispersion = m.dispersion;
    r.metallic = m.metallic;
    r.alphaCutoff = m.alpha_cutoff;
    r.alphaMasked = m.alpha_masked != 0;
    r.attenuationColor = v3(m.attenuation_color);
    r.attenuationDistance = m.attenuation_distance;
    r.volumeDensity = m.volume_density;
    r.specular = v3(m.specular);
    r.glossiness = m.glossiness;
    r.opacity = m.opacity;
    r.specularGlossinessWorkflow = m.specgloss_workflow != 0;
    r.gltfPbrWorkflow = m.gltf_pbr != 0;
    r.specularWeight = m.specular_weight;
    r.specularColor = v3(m.specular_color);
    r.clearcoat = m.clearcoat;
    r.clearcoatRoughness = m.clearcoat_roughness;
    return r;
}

// probe: the hit-identity probe copy (light registration off, triangle
// lightIndex = identity code, material overrides baked into per-instance
// mesh copies, one private material per sphere); the instance light offsets
// are set by the caller after uploadScene.
inline void host_scene_from_desc(const wf_scene_desc* d, bool probe, HostScene& h) {
    for (uint32_t i = 0; i < d->material_count; ++i) {
        h.materials.push_back(to_material(d->materials[i]));
        if (d->material_textures) apply_textures(h.materials.back(), d->material_textures[i]);
    }
    for (uint32_t i = 0; i < d->texture_count; ++i) {
        const wf_texture& t = d->textures[i];
        ObjTexture o;
        o.width = t.width;
        o.height = t.height;
        o.pixels.assign(t.rgba, t.rgba + size_t(t.width) * t.height * 4);
        h.textures.push_back(std::move(o));
    }
    for (uint32_t i = 0; i < d->sphere_count; ++i) {
        const wf_sphere& s = d->spheres[i];
        uint32_t material = s.material;
        if (probe) {
            material = uint32_t(h.materials.size());
            h.materials.push_back(h.materials.at(s.material));
        }
        h.spheres.emplace_back(Sphere{v3(s.center), s.radius, material},
                               s.accel == WF_ACCEL_DIRECT ? AccelerationMode::Direct : AccelerationMode::Bvh);
    }
    for (uint32_t i = 0; i < d->triangle_count; ++i) {
        h.triangles.push_back(to_triangle(d->triangles[i], d->triangle_attributes ? &d->triangle_attributes[i] : nullptr));
        if (probe) h.triangles.back().lightIndex = 0x80000000u | i;
    }
    for (uint32_t i = 0; i < d->static_triangle_count; ++i) {
        h.staticTriangles.push_back(
            to_triangle(d->static_triangles[i], d->static_triangle_attributes ? &d->static_triangle_attributes[i] : nullptr));
        if (probe) h.staticTriangles.back().lightIndex = 0x40000000u | i;
    }
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        MeshAsset mesh;
        for (uint32_t i = 0; i < d->meshes[m].triangle_count; ++i) {
            mesh.triangles.push_back(
                to_triangle(d->meshes[m].triangles[i], d->meshes[m].attributes ? &d->meshes[m].attributes[i] : nullptr));
            if (probe) mesh.triangles.back().lightIndex = i;
        }
        h.meshes.push_back(std::move(mesh));
    }
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const wf_instance& in = d->instances[i];
        InstanceTransform t;
        t.localToWorldX = v3(in.local_to_world[0]);
        t.localToWorldY = v3(in.local_to_world[1]);
        t.localToWorldZ = v3(in.local_to_world[2]);
        t.worldToLocalX = v3(in.world_to_local[0]);
        t.worldToLocalY = v3(in.world_to_local[1]);
        t.worldToLocalZ = v3(in.world_to_local[2]);
        t.translation = v3(in.translation);
        uint32_t mesh = in.mesh;
        uint32_t override_material = in.material_override;
        if (probe && override_material != invalidMaterialIndex) {
            // The override would hide the triangle's identity code
            // (lightIndex is dropped for overridden instances): bake it
            // into a private copy of the mesh instead.  Same positions,
            // so the builder produces the same tree.
            MeshAsset copy = h.meshes[in.mesh];
            for (Triangle& tri : copy.triangles) tri.material = override_material;
            mesh = uint32_t(h.meshes.size());
            h.meshes.push_back(std::move(copy));
            override_material = invalidMaterialIndex;
        }
        SceneInstance si{mesh, t, override_material,
                         in.accel == WF_ACCEL_DIRECT ? AccelerationMode::Direct : AccelerationMode::Bvh};
        h.instances.push_back(si);
    }
    for (uint32_t i = 0; i < d->punctual_light_count; ++i) {
        const wf_punctual_light& l = d->punctual_lights[i];
        PunctualLight p;
        p.type = PunctualLightType(l.type);
        p.position = v3(l.position);
        p.direction = v3(l.direction);
        p.intensity = v3(l.intensity);
        p.range = l.range;
        p.innerConeCos = l.inner_cone_cos;
        p.outerConeCos = l.outer_cone_cos;
        h.punctualLights.push_back(p);
    }
    h.blackBackground = d->black_background != 0;
    h.acceleration = ObjAccelerationPolicy::NexusBvh2;
    if (d->register_triangle_lights && !probe) wfref_register_lights(h);
}

}  // namespace wfref
