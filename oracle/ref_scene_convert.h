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

inline Triangle to_triangle(const wf_triangle& t) {
    Triangle r{};
    r.v0 = v3(t.v0); r.v1 = v3(t.v1); r.v2 = v3(t.v2);
    r.n0 = v3(t.n0); r.n1 = v3(t.n1); r.n2 = v3(t.n2);
    r.material = t.material;
    r.lightIndex = invalidLightIndex;
    r.hasVertexNormals = t.has_vertex_normals != 0;
    return r;
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
    for (uint32_t i = 0; i < d->material_count; ++i) h.materials.push_back(to_material(d->materials[i]));
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
        h.triangles.push_back(to_triangle(d->triangles[i]));
        if (probe) h.triangles.back().lightIndex = 0x80000000u | i;
    }
    for (uint32_t i = 0; i < d->static_triangle_count; ++i) {
        h.staticTriangles.push_back(to_triangle(d->static_triangles[i]));
        if (probe) h.staticTriangles.back().lightIndex = 0x40000000u | i;
    }
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        MeshAsset mesh;
        for (uint32_t i = 0; i < d->meshes[m].triangle_count; ++i) {
            mesh.triangles.push_back(to_triangle(d->meshes[m].triangles[i]));
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
