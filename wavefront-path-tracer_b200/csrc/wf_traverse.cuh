// Closest-hit and any-hit traversal.
//
// Semantics follow the reference's traceRay / isOccluded
// (include/renderer/device_traversal.cuh:1035-1184) exactly: the same visit
// order (direct spheres, direct instances, static triangles, TLAS, direct
// triangle list), the same slab and Moller-Trumbore arithmetic, the same
// strict "<" tie rule for triangles and lower-index rule for spheres, and the
// same near-first child order (ties go to the right child).  The node layout
// differs (both child boxes in the parent, see wf_device.cuh); a popped entry
// carries the entry distance recorded when it was pushed, and re-testing
// "entry < closestT" is exactly the reference's re-test of the popped node's
// box (its other condition cannot change between push and pop).
#pragma once

#include <cfloat>

#include "wf_device.cuh"

namespace wf {

constexpr int kStackSize = 64;  // leaf depth <= kMaxBvhDepth (60) < 64

// Traversal work tallies.  NoTally compiles away; CountTally records the
// node visits (one visit = one 64-byte node = two child boxes), triangle,
// sphere and instance tests a traversal performs, for the algorithmic-byte
// accounting of the profiling pass.
// A tally type also fixes, at compile time, whether the traversal may meet
// alpha-textured materials (kAlphaTextures): the default types handle every
// scene; Opaque<T> compiles the per-hit texture test out, for kernels that
// the host launches only on scenes without such materials.
struct NoTally {
    static constexpr bool kCounts = false;
    static constexpr bool kAlphaTextures = true;
    WF_DEV void node() {}
    WF_DEV void triangle() {}
    WF_DEV void sphere() {}
    WF_DEV void instance() {}
};
struct CountTally {
    static constexpr bool kCounts = true;
    static constexpr bool kAlphaTextures = true;
    uint32_t nodes = 0, triangles = 0, spheres = 0, instances = 0;
    WF_DEV void node() { ++nodes; }
    WF_DEV void triangle() { ++triangles; }
    WF_DEV void sphere() { ++spheres; }
    WF_DEV void instance() { ++instances; }
};
template <typename Base>
struct Opaque : Base {
    static constexpr bool kAlphaTextures = false;
};

struct TraceState {
    float t;          // closestT
    float u, v;
    uint32_t prim;    // make_prim(kind, index); kind kHitMiss = no hit
    uint32_t inst;    // instance of a kHitMesh hit
    uint32_t sphere;  // closestSphereIndex (reset to kInvalid by triangle hits)
};

WF_DEV void trace_state_init(TraceState& h, float t_max) {
    h.t = t_max;
    h.u = h.v = 0.0f;
    h.prim = make_prim(kHitMiss, 0);
    h.inst = kInvalid;
    h.sphere = kInvalid;
}

// intersectAabb, device_traversal.cuh:182-197.
WF_DEV bool slab(V3 o, V3 inv, float lox, float hix, float loy, float hiy, float loz, float hiz,
                 float closest_t, float& near_t) {
    float tx0 = (lox - o.x) * inv.x;
    float tx1 = (hix - o.x) * inv.x;
    float ty0 = (loy - o.y) * inv.y;
    float ty1 = (hiy - o.y) * inv.y;
    float tz0 = (loz - o.z) * inv.z;
    float tz1 = (hiz - o.z) * inv.z;
    float tmin = fmaxf(fminf(tx0, tx1), fmaxf(fminf(ty0, ty1), fminf(tz0, tz1)));
    float tmax = fminf(fmaxf(tx0, tx1), fminf(fmaxf(ty0, ty1), fmaxf(tz0, tz1)));
    near_t = tmin;
    return tmax >= fmaxf(tmin, kRayMinDistance) && tmin < closest_t;
}

WF_DEV bool slab_box(V3 o, V3 inv, const Box& b, float closest_t, float& near_t) {
    return slab(o, inv, b.lo[0], b.hi[0], b.lo[1], b.hi[1], b.lo[2], b.hi[2], closest_t, near_t);
}

WF_DEV V3 inverse_direction(V3 d) { return V3{1.0f / d.x, 1.0f / d.y, 1.0f / d.z}; }

// intersectSphere, device_traversal.cuh:24-53.
WF_DEV bool intersect_sphere(V3 o, V3 d, float4 s, float& t) {
    V3 oc = o - V3{s.x, s.y, s.z};
    float a = dot(d, d);
    float b = 2.0f * dot(oc, d);
    float c = dot(oc, oc) - s.w * s.w;
    float discriminant = b * b - 4.0f * a * c;
    if (discriminant < 0.0f) return false;
    float sq = sqrtf(discriminant);
    float t0 = (-b - sq) / (2.0f * a);
    float t1 = (-b + sq) / (2.0f * a);
    if (t0 > kRayMinDistance) { t = t0; return true; }
    if (t1 > kRayMinDistance) { t = t1; return true; }
    return false;
}

// intersectTriangle, device_traversal.cuh:55-91 (Moller-Trumbore with the
// determinant-scale cancellation guard).
WF_DEV bool intersect_triangle(V3 o, V3 d, V3 v0, V3 v1, V3 v2, float& t, float& u, float& v) {
    V3 e1 = v1 - v0;
    V3 e2 = v2 - v0;
    V3 p = cross(d, e2);
    float det = dot(e1, p);
    float scale = fabsf(e1.x) * (fabsf(d.y * e2.z) + fabsf(d.z * e2.y)) +
                  fabsf(e1.y) * (fabsf(d.z * e2.x) + fabsf(d.x * e2.z)) +
                  fabsf(e1.z) * (fabsf(d.x * e2.y) + fabsf(d.y * e2.x));
    if (!isfinite(det) || fabsf(det) <= 8.0f * FLT_EPSILON * scale) return false;
    float inv = 1.0f / det;
    V3 ov = o - v0;
    u = dot(ov, p) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    V3 q = cross(ov, e1);
    v = dot(d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, q) * inv;
    return t > kRayMinDistance;
}

struct TriVerts {
    V3 v0, v1, v2;
    uint32_t index_flags, material, light;
};

WF_DEV TriVerts load_triangle(const DeviceScene& s, uint32_t i) {
    float4 a = __ldg(&s.triangles[3 * size_t(i)]);
    float4 b = __ldg(&s.triangles[3 * size_t(i) + 1]);
    float4 c = __ldg(&s.triangles[3 * size_t(i) + 2]);
    return TriVerts{f4xyz(a), f4xyz(b), f4xyz(c), __float_as_uint(a.w), __float_as_uint(b.w),
                    __float_as_uint(c.w)};
}

// ---------------------------------------------------------------- textures
// tex2D<float4> on an RGBA8 texture with normalised reads, wrap addressing
// and linear filtering (src/scene/scene.cu:54-69), in the arithmetic of the
// host replay of the reference's kernels (cpu_replay.cpp:14-24): texel-centre
// offset, floor, wrap, weights (1 - f, f), rows then columns, bytes / 255 as
// bytes * (1 / 255).
WF_DEV float4 texture_fetch(const DeviceScene& s, uint32_t texture, float u, float v) {
    uint4 info = s.textures[texture];
    int w = int(info.x), h = int(info.y);
    float tx = u * float(info.x) - .5f, ty = v * float(info.y) - .5f;
    int x = int(floorf(tx)), y = int(floorf(ty));
    float fx = tx - float(x), fy = ty - float(y);
    const float scale = 1.0f / 255.0f;
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            int xx = (((x + i) % w) + w) % w, yy = (((y + j) % h) + h) % h;
            uchar4 p = s.texels[info.z + size_t(yy) * uint32_t(w) + uint32_t(xx)];
            float wt = (i ? fx : 1.0f - fx) * (j ? fy : 1.0f - fy);
            r.x += wt * (float(p.x) * scale);
            r.y += wt * (float(p.y) * scale);
            r.z += wt * (float(p.z) * scale);
            r.w += wt * (float(p.w) * scale);
        }
    return r;
}

// getTriangleUv, device_traversal.cuh:120-131, for both coordinate sets.
WF_DEV void triangle_uvs(const DeviceScene& s, uint32_t ti, float u, float v, float2& uv, float2& uv1) {
    uv = uv1 = make_float2(0.0f, 0.0f);
    if (!s.tri_attr) return;
    const TriAttr& a = s.tri_attr[ti];
    float w = 1.0f - u - v;
    if (a.has_texcoords)
        uv = make_float2(w * a.uv[0][0] + u * a.uv[1][0] + v * a.uv[2][0], w * a.uv[0][1] + u * a.uv[1][1] + v * a.uv[2][1]);
    if (a.has_texcoords1)
        uv1 = make_float2(w * a.uv1[0][0] + u * a.uv1[1][0] + v * a.uv1[2][0],
                          w * a.uv1[0][1] + u * a.uv1[1][1] + v * a.uv1[2][1]);
}

// getTextureUv + sampleTexture, device_traversal.cuh:325-347.
WF_DEV float4 sample_binding(const DeviceScene& s, const TexBinding& b, float2 uv, float2 uv1, float4 fallback) {
    if (b.texture == kInvalid || b.texture >= s.texture_count) return fallback;
    float2 t = b.texcoord == 1 ? uv1 : uv;
    if (b.has_transform) {
        t.x *= b.scale_x;
        t.y *= b.scale_y;
        float sine = wfm::sinf(b.rotation), cosine = wfm::cosf(b.rotation);
        t = make_float2(cosine * t.x - sine * t.y + b.offset_x, sine * t.x + cosine * t.y + b.offset_y);
    }
    return texture_fetch(s, b.texture, t.x, 1.0f - t.y);
}

// alphaMasked && getMaterialOpacity < alphaCutoff (device_traversal.cuh:
// 150,265,370-378): untextured materials carry the answer as a flag; with an
// albedo texture the opacity is read at the candidate hit.  Tally decides at
// compile time whether the texture test exists in the kernel.
template <typename Tally>
WF_DEV bool alpha_rejects(const DeviceScene& s, uint32_t material, uint32_t ti, float u, float v) {
    if (!s.any_alpha_reject) return false;
    uint32_t flags = s.materials[material].flags;
    if constexpr (Tally::kAlphaTextures) {
        if (flags & kMatAlphaTexture) {
            const MaterialTextures& mt = s.material_textures[material];
            float2 uv, uv1;
            triangle_uvs(s, ti, u, v, uv, uv1);
            float opacity =
                mt.opacity * sample_binding(s, mt.slot[kTexAlbedo], uv, uv1, make_float4(1.0f, 1.0f, 1.0f, 1.0f)).w;
            return opacity < mt.alpha_cutoff;
        }
    }
    return (flags & kMatAlphaReject) != 0;
}

// Local stack of (ref, entry distance).
struct Stack {
    int ref[kStackSize];
    float t[kStackSize];
    int size;
};

// Closest hit in one BVH over triangles (BLAS with a local ray, or the direct
// list with the world ray).  intersectNexusBvh2, device_traversal.cuh:239-313.
// kind/inst label accepted hits; override replaces the triangle material.
template <typename Tally>
WF_DEV void bvh_closest(const DeviceScene& s, const BvhRef& bvh, V3 o, V3 d, TraceState& h,
                        uint32_t kind, uint32_t inst, uint32_t material_override, Tally& tally) {
    V3 inv = inverse_direction(d);
    float near_t;
    if (bvh.root == kNoRoot || !slab_box(o, inv, bvh.box, h.t, near_t)) return;
    Stack st;
    st.size = 0;
    int ref = bvh.root;
    for (;;) {
        if (ref < 0) {
            uint32_t ti = uint32_t(~ref);
            tally.triangle();
            TriVerts tri = load_triangle(s, ti);
            float t, u, v;
            if (intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) && t < h.t) {
                uint32_t m = material_override == kInvalid ? tri.material : material_override;
                if (!alpha_rejects<Tally>(s, m, ti, u, v)) {
                    h.t = t;
                    h.u = u;
                    h.v = v;
                    h.prim = make_prim(kind, ti);
                    h.inst = inst;
                }
            }
        } else {
            tally.node();
            const BvhNode* node = &s.nodes[ref];
            float4 lxy = __ldg(&node->lxy);
            float4 rxy = __ldg(&node->rxy);
            float4 lrz = __ldg(&node->lrz);
            int4 ch = __ldg(&node->child);
            float tl, tr;
            bool hl = slab(o, inv, lxy.x, lxy.y, lxy.z, lxy.w, lrz.x, lrz.y, h.t, tl);
            bool hr = slab(o, inv, rxy.x, rxy.y, rxy.z, rxy.w, lrz.z, lrz.w, h.t, tr);
            if (hl && hr) {
                bool left_near = tl < tr;
                if (st.size < kStackSize) {  // depth <= kMaxBvhDepth < kStackSize by construction
                    st.ref[st.size] = left_near ? ch.y : ch.x;
                    st.t[st.size] = left_near ? tr : tl;
                    ++st.size;
                }
                ref = left_near ? ch.x : ch.y;
                continue;
            }
            if (hl) { ref = ch.x; continue; }
            if (hr) { ref = ch.y; continue; }
        }
        for (;;) {
            if (st.size == 0) return;
            --st.size;
            if (st.t[st.size] < h.t) break;
        }
        ref = st.ref[st.size];
    }
}

// Any hit with t < t_max in one triangle BVH.
template <typename Tally>
WF_DEV bool bvh_any(const DeviceScene& s, const BvhRef& bvh, V3 o, V3 d, float t_max,
                    uint32_t material_override, Tally& tally) {
    V3 inv = inverse_direction(d);
    float near_t;
    if (bvh.root == kNoRoot || !slab_box(o, inv, bvh.box, t_max, near_t)) return false;
    int stack[kStackSize];
    int size = 0;
    int ref = bvh.root;
    for (;;) {
        if (ref < 0) {
            uint32_t ti = uint32_t(~ref);
            tally.triangle();
            TriVerts tri = load_triangle(s, ti);
            float t, u, v;
            if (intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) && t < t_max) {
                uint32_t m = material_override == kInvalid ? tri.material : material_override;
                if (!alpha_rejects<Tally>(s, m, ti, u, v)) return true;
            }
        } else {
            tally.node();
            const BvhNode* node = &s.nodes[ref];
            float4 lxy = __ldg(&node->lxy);
            float4 rxy = __ldg(&node->rxy);
            float4 lrz = __ldg(&node->lrz);
            int4 ch = __ldg(&node->child);
            float tl, tr;
            bool hl = slab(o, inv, lxy.x, lxy.y, lxy.z, lxy.w, lrz.x, lrz.y, t_max, tl);
            bool hr = slab(o, inv, rxy.x, rxy.y, rxy.z, rxy.w, lrz.z, lrz.w, t_max, tr);
            if (hl && hr) {
                bool left_near = tl < tr;
                if (size < kStackSize) stack[size++] = left_near ? ch.y : ch.x;
                ref = left_near ? ch.x : ch.y;
                continue;
            }
            if (hl) { ref = ch.x; continue; }
            if (hr) { ref = ch.y; continue; }
        }
        if (size == 0) return false;
        ref = stack[--size];
    }
}

// inverseTransformVector(T, v), include/scene/scene.cuh:44-47.
WF_DEV V3 to_local_vector(const Instance& in, V3 v) {
    V3 x{in.w2l_x.x, in.w2l_x.y, in.w2l_x.z};
    V3 y{in.w2l_y.x, in.w2l_y.y, in.w2l_y.z};
    V3 z{in.w2l_z.x, in.w2l_z.y, in.w2l_z.z};
    return x * v.x + y * v.y + z * v.z;
}
WF_DEV V3 instance_translation(const Instance& in) { return V3{in.w2l_x.w, in.w2l_y.w, in.w2l_z.w}; }

WF_DEV Instance load_instance(const DeviceScene& s, uint32_t i) {
    const Instance* p = &s.instances[i];
    Instance in;
    in.w2l_x = __ldg(&p->w2l_x);
    in.w2l_y = __ldg(&p->w2l_y);
    in.w2l_z = __ldg(&p->w2l_z);
    in.blas = __ldg(&p->blas);
    in.light_offset = __ldg(&p->light_offset);
    in.material_override = __ldg(&p->material_override);
    return in;
}

// Linear scan of a mesh in original triangle order (intersectMeshInstance
// with useBvh = false, device_traversal.cuh:814-821).
template <typename Tally>
WF_DEV void mesh_linear_closest(const DeviceScene& s, const Blas& b, V3 o, V3 d, TraceState& h,
                                uint32_t inst, uint32_t material_override, Tally& tally) {
    for (uint32_t i = 0; i < b.count; ++i) {
        uint32_t ti = s.mesh_linear[b.first_linear + i];
        tally.triangle();
        TriVerts tri = load_triangle(s, ti);
        float t, u, v;
        if (!intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) || t >= h.t) continue;
        uint32_t m = material_override == kInvalid ? tri.material : material_override;
        if (alpha_rejects<Tally>(s, m, ti, u, v)) continue;
        h.t = t;
        h.u = u;
        h.v = v;
        h.prim = make_prim(kHitMesh, ti);
        h.inst = inst;
    }
}

// intersectMeshInstance, device_traversal.cuh:802-834 (attribute transforms
// are deferred to finish_hit).
template <typename Tally>
WF_DEV void instance_closest(const DeviceScene& s, uint32_t inst, V3 o, V3 d, TraceState& h, bool use_bvh, Tally& tally) {
    tally.instance();
    Instance in = load_instance(s, inst);
    Blas b = s.blases[in.blas];
    V3 lo = to_local_vector(in, o - instance_translation(in));
    V3 ld = to_local_vector(in, d);
    float previous = h.t;
    if (use_bvh && b.bvh.root != kNoRoot)
        bvh_closest(s, b.bvh, lo, ld, h, kHitMesh, inst, in.material_override, tally);
    else
        mesh_linear_closest(s, b, lo, ld, h, inst, in.material_override, tally);
    if (h.t >= previous) return;
    h.sphere = kInvalid;
}

template <typename Tally>
WF_DEV bool instance_any(const DeviceScene& s, uint32_t inst, V3 o, V3 d, float t_max, bool use_bvh, Tally& tally) {
    tally.instance();
    Instance in = load_instance(s, inst);
    Blas b = s.blases[in.blas];
    V3 lo = to_local_vector(in, o - instance_translation(in));
    V3 ld = to_local_vector(in, d);
    if (use_bvh && b.bvh.root != kNoRoot) return bvh_any(s, b.bvh, lo, ld, t_max, in.material_override, tally);
    for (uint32_t i = 0; i < b.count; ++i) {
        tally.triangle();
        TriVerts tri = load_triangle(s, s.mesh_linear[b.first_linear + i]);
        float t, u, v;
        if (!intersect_triangle(lo, ld, tri.v0, tri.v1, tri.v2, t, u, v) || t >= t_max) continue;
        uint32_t m = in.material_override == kInvalid ? tri.material : in.material_override;
        if (!alpha_rejects<Tally>(s, m, s.mesh_linear[b.first_linear + i], u, v)) return true;
    }
    return false;
}

// intersectSphereHit, device_traversal.cuh:789-800.
template <typename Tally>
WF_DEV void sphere_closest(const DeviceScene& s, uint32_t index, V3 o, V3 d, TraceState& h, Tally& tally) {
    float t;
    tally.sphere();
    if (!intersect_sphere(o, d, __ldg(&s.spheres[index]), t) || t > h.t) return;
    if (t == h.t && index >= h.sphere) return;
    h.t = t;
    h.prim = make_prim(kHitSphere, index);
    h.sphere = index;
}

// intersectSceneTlas, device_traversal.cuh:836-878.
template <typename Tally>
WF_DEV void tlas_closest(const DeviceScene& s, V3 o, V3 d, TraceState& h, Tally& tally) {
    if (s.tlas.root == kNoRoot) return;
    V3 inv = inverse_direction(d);
    float near_t;
    if (!slab_box(o, inv, s.tlas.box, h.t, near_t)) return;
    Stack st;
    st.size = 0;
    int ref = s.tlas.root;
    for (;;) {
        if (ref < 0) {
            uint32_t leaf = __ldg(&s.tlas_leaves[~ref]);
            if (leaf & 0x80000000u)
                sphere_closest(s, leaf & 0x7fffffffu, o, d, h, tally);
            else
                instance_closest(s, leaf, o, d, h, true, tally);
        } else {
            tally.node();
            const BvhNode* node = &s.nodes[ref];
            float4 lxy = __ldg(&node->lxy);
            float4 rxy = __ldg(&node->rxy);
            float4 lrz = __ldg(&node->lrz);
            int4 ch = __ldg(&node->child);
            float tl, tr;
            bool hl = slab(o, inv, lxy.x, lxy.y, lxy.z, lxy.w, lrz.x, lrz.y, h.t, tl);
            bool hr = slab(o, inv, rxy.x, rxy.y, rxy.z, rxy.w, lrz.z, lrz.w, h.t, tr);
            if (hl && hr) {
                bool left_near = tl < tr;
                if (st.size < kStackSize) {  // depth <= kMaxBvhDepth < kStackSize by construction
                    st.ref[st.size] = left_near ? ch.y : ch.x;
                    st.t[st.size] = left_near ? tr : tl;
                    ++st.size;
                }
                ref = left_near ? ch.x : ch.y;
                continue;
            }
            if (hl) { ref = ch.x; continue; }
            if (hr) { ref = ch.y; continue; }
        }
        for (;;) {
            if (st.size == 0) return;
            --st.size;
            if (st.t[st.size] < h.t) break;
        }
        ref = st.ref[st.size];
    }
}

template <typename Tally>
WF_DEV bool tlas_any(const DeviceScene& s, V3 o, V3 d, float t_max, Tally& tally) {
    if (s.tlas.root == kNoRoot) return false;
    V3 inv = inverse_direction(d);
    float near_t;
    if (!slab_box(o, inv, s.tlas.box, t_max, near_t)) return false;
    int stack[kStackSize];
    int size = 0;
    int ref = s.tlas.root;
    for (;;) {
        if (ref < 0) {
            uint32_t leaf = __ldg(&s.tlas_leaves[~ref]);
            if (leaf & 0x80000000u) {
                float t;
                tally.sphere();
                if (intersect_sphere(o, d, __ldg(&s.spheres[leaf & 0x7fffffffu]), t) && t < t_max) return true;
            } else if (instance_any(s, leaf, o, d, t_max, true, tally)) {
                return true;
            }
        } else {
            tally.node();
            const BvhNode* node = &s.nodes[ref];
            float4 lxy = __ldg(&node->lxy);
            float4 rxy = __ldg(&node->rxy);
            float4 lrz = __ldg(&node->lrz);
            int4 ch = __ldg(&node->child);
            float tl, tr;
            bool hl = slab(o, inv, lxy.x, lxy.y, lxy.z, lxy.w, lrz.x, lrz.y, t_max, tl);
            bool hr = slab(o, inv, rxy.x, rxy.y, rxy.z, rxy.w, lrz.z, lrz.w, t_max, tr);
            if (hl && hr) {
                bool left_near = tl < tr;
                if (size < kStackSize) stack[size++] = left_near ? ch.y : ch.x;
                ref = left_near ? ch.x : ch.y;
                continue;
            }
            if (hl) { ref = ch.x; continue; }
            if (hr) { ref = ch.y; continue; }
        }
        if (size == 0) return false;
        ref = stack[--size];
    }
}

// traceRay, device_traversal.cuh:1115-1150 (visit order and sphere reset rules).
template <typename Tally>
WF_DEV void trace_closest(const DeviceScene& s, V3 o, V3 d, TraceState& h, Tally& tally) {
    trace_state_init(h, 1e30f);
    for (uint32_t i = 0; i < s.direct_sphere_count; ++i) sphere_closest(s, s.direct_spheres[i], o, d, h, tally);
    for (uint32_t i = 0; i < s.direct_instance_count; ++i) instance_closest(s, s.direct_instances[i], o, d, h, false, tally);
    for (uint32_t i = 0; i < s.static_count; ++i) {
        uint32_t ti = s.static_first + i;
        tally.triangle();
        TriVerts tri = load_triangle(s, ti);
        float t, u, v;
        if (!intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) || t >= h.t) continue;
        if (alpha_rejects<Tally>(s, tri.material, ti, u, v)) continue;
        h.t = t;
        h.u = u;
        h.v = v;
        h.prim = make_prim(kHitTriangle, ti);
        h.inst = kInvalid;
        h.sphere = kInvalid;
    }
    tlas_closest(s, o, d, h, tally);
    if (s.direct_count > 0) {
        float previous = h.t;
        if (s.direct_bvh.root != kNoRoot) {
            bvh_closest(s, s.direct_bvh, o, d, h, kHitTriangle, kInvalid, kInvalid, tally);
        } else {
            for (uint32_t i = 0; i < s.direct_count; ++i) {
                uint32_t ti = s.direct_first + i;
                tally.triangle();
                TriVerts tri = load_triangle(s, ti);
                float t, u, v;
                if (!intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) || t >= h.t) continue;
                if (alpha_rejects<Tally>(s, tri.material, ti, u, v)) continue;
                h.t = t;
                h.u = u;
                h.v = v;
                h.prim = make_prim(kHitTriangle, ti);
                h.inst = kInvalid;
            }
        }
        if (h.t < previous) h.sphere = kInvalid;
    }
}

// isOccluded, device_traversal.cuh:1035-1113.  A pure disjunction of
// independent tests, so an early return at the first hit gives the same bit.
template <typename Tally>
WF_DEV bool trace_any(const DeviceScene& s, V3 o, V3 d, float t_max, Tally& tally) {
    for (uint32_t i = 0; i < s.direct_sphere_count; ++i) {
        float t;
        tally.sphere();
        if (intersect_sphere(o, d, __ldg(&s.spheres[s.direct_spheres[i]]), t) && t < t_max) return true;
    }
    for (uint32_t i = 0; i < s.direct_instance_count; ++i)
        if (instance_any(s, s.direct_instances[i], o, d, t_max, false, tally)) return true;
    for (uint32_t i = 0; i < s.static_count; ++i) {
        tally.triangle();
        TriVerts tri = load_triangle(s, s.static_first + i);
        float t, u, v;
        if (intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) && t < t_max &&
            !alpha_rejects<Tally>(s, tri.material, s.static_first + i, u, v))
            return true;
    }
    if (tlas_any(s, o, d, t_max, tally)) return true;
    if (s.direct_count > 0) {
        if (s.direct_bvh.root != kNoRoot) return bvh_any(s, s.direct_bvh, o, d, t_max, kInvalid, tally);
        for (uint32_t i = 0; i < s.direct_count; ++i) {
            tally.triangle();
            TriVerts tri = load_triangle(s, s.direct_first + i);
            float t, u, v;
            if (intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) && t < t_max &&
                !alpha_rejects<Tally>(s, tri.material, s.direct_first + i, u, v))
                return true;
        }
    }
    return false;
}

// Surface attributes of the winning primitive (the Hit fields the shading
// stage uses), computed once after traversal exactly as the reference
// computes them at acceptance time: getTriangleGeometricNormal /
// getTriangleNormal with the (local) ray, transformNormal for instances
// (device_traversal.cuh:104-125,149-152,824-832; scene.cuh:50-55), sphere
// normals at the end of traceRay (:1152-1160).
struct SurfaceHit {
    float t;
    V3 position;
    V3 geometric_normal;
    V3 normal;
    uint32_t material;
    uint32_t light;
    // texture coordinates and tangent frames (Hit::uv .. bitangent1); zero
    // for spheres and for scenes without triangle attributes
    float2 uv, uv1;
    V3 tangent, bitangent, tangent1, bitangent1;
};

// transformVector, include/scene/scene.cuh:40-42.
WF_DEV V3 transform_vector(const Instance& in, V3 v) {
    return V3{in.l2w_x.x, in.l2w_x.y, in.l2w_x.z} * v.x + V3{in.l2w_y.x, in.l2w_y.y, in.l2w_y.z} * v.y +
           V3{in.l2w_z.x, in.l2w_z.y, in.l2w_z.z} * v.z;
}

// The texture coordinates and tangent frame intersectTriangleHit records for
// the winning triangle (device_traversal.cuh:147-174), with `n` its
// (face-forwarded, instance-local) shading normal.
WF_DEV void triangle_frames(const DeviceScene& s, uint32_t ti, float u, float v, V3 n, SurfaceHit& out) {
    triangle_uvs(s, ti, u, v, out.uv, out.uv1);
    const TriAttr& a = s.tri_attr[ti];
    V3 tangent{a.tangent[0], a.tangent[1], a.tangent[2]};
    V3 bitangent{a.bitangent[0], a.bitangent[1], a.bitangent[2]};
    if (a.has_vertex_tangents) {
        float w = 1.0f - u - v;
        V3 t = w * V3{a.vertex_tangent[0][0], a.vertex_tangent[0][1], a.vertex_tangent[0][2]} +
               u * V3{a.vertex_tangent[1][0], a.vertex_tangent[1][1], a.vertex_tangent[1][2]} +
               v * V3{a.vertex_tangent[2][0], a.vertex_tangent[2][1], a.vertex_tangent[2][2]};
        t = t - n * dot(n, t);
        if (length_squared(t) > 0.00000001f) {
            tangent = normalize(t);
            float sign = w * a.vertex_tangent_sign[0] + u * a.vertex_tangent_sign[1] + v * a.vertex_tangent_sign[2];
            bitangent = (sign < 0.0f ? -1.0f : 1.0f) * normalize(cross(n, tangent));
        }
    }
    out.tangent = tangent;
    out.bitangent = bitangent;
    out.tangent1 = V3{a.tangent1[0], a.tangent1[1], a.tangent1[2]};
    out.bitangent1 = V3{a.bitangent1[0], a.bitangent1[1], a.bitangent1[2]};
}

WF_DEV V3 triangle_geometric_normal(const TriVerts& tri, V3 d, bool face_forward) {
    V3 n = normalize(cross(tri.v1 - tri.v0, tri.v2 - tri.v0));
    return face_forward && dot(n, d) > 0.0f ? -n : n;
}

WF_DEV V3 triangle_shading_normal(const DeviceScene& s, uint32_t ti, const TriVerts& tri, V3 d, float u,
                                  float v, bool face_forward) {
    V3 n;
    if ((tri.index_flags & kTriHasNormals) && s.normals) {
        V3 n0 = f4xyz(s.normals[3 * size_t(ti)]);
        V3 n1 = f4xyz(s.normals[3 * size_t(ti) + 1]);
        V3 n2 = f4xyz(s.normals[3 * size_t(ti) + 2]);
        n = normalize((1.0f - u - v) * n0 + u * n1 + v * n2);
    } else {
        n = normalize(cross(tri.v1 - tri.v0, tri.v2 - tri.v0));
    }
    return face_forward && dot(n, d) > 0.0f ? -n : n;
}

// transformNormal, include/scene/scene.cuh:50-55.
WF_DEV V3 transform_normal(const Instance& in, V3 n) {
    V3 x{in.w2l_x.x, in.w2l_x.y, in.w2l_x.z};
    V3 y{in.w2l_y.x, in.w2l_y.y, in.w2l_y.z};
    V3 z{in.w2l_z.x, in.w2l_z.y, in.w2l_z.z};
    return normalize(V3{dot(x, n), dot(y, n), dot(z, n)});
}

WF_DEV bool finish_hit(const DeviceScene& s, V3 o, V3 d, float t, float u, float v, uint32_t prim,
                       uint32_t inst, SurfaceHit& out) {
    uint32_t kind = hit_kind(prim), index = hit_index(prim);
    if (kind == kHitMiss) return false;
    out.t = t;
    out.uv = out.uv1 = make_float2(0.0f, 0.0f);
    out.tangent = out.bitangent = out.tangent1 = out.bitangent1 = V3{0.0f, 0.0f, 0.0f};
    if (kind == kHitSphere) {
        float4 sp = __ldg(&s.spheres[index]);
        V3 at = o + d * t;
        out.normal = normalize(at - V3{sp.x, sp.y, sp.z});
        out.geometric_normal = out.normal;
        out.material = s.sphere_materials[index];
        out.light = kInvalid;
    } else if (kind == kHitTriangle) {
        TriVerts tri = load_triangle(s, index);
        out.material = tri.material;
        bool ff = s.materials[tri.material].type != kDielectric;
        out.geometric_normal = triangle_geometric_normal(tri, d, ff);
        out.normal = triangle_shading_normal(s, index, tri, d, u, v, ff);
        out.light = tri.light;
        if (s.tri_attr) triangle_frames(s, index, u, v, out.normal, out);
    } else {
        Instance in = load_instance(s, inst);
        TriVerts tri = load_triangle(s, index);
        V3 ld = to_local_vector(in, d);
        uint32_t m = in.material_override == kInvalid ? tri.material : in.material_override;
        out.material = m;
        bool ff = s.materials[m].type != kDielectric;
        V3 gn = triangle_geometric_normal(tri, ld, ff);
        V3 n = triangle_shading_normal(s, index, tri, ld, u, v, ff);
        out.geometric_normal = transform_normal(in, gn);
        out.normal = transform_normal(in, n);
        if (s.tri_attr) {  // intersectMeshInstance, device_traversal.cuh:826-829
            triangle_frames(s, index, u, v, n, out);
            const Instance& full = s.instances[inst];  // load_instance reads only the world-to-local rows
            out.tangent = normalize(transform_vector(full, out.tangent));
            out.bitangent = normalize(transform_vector(full, out.bitangent));
            out.tangent1 = normalize(transform_vector(full, out.tangent1));
            out.bitangent1 = normalize(transform_vector(full, out.bitangent1));
        }
        uint32_t light = in.material_override == kInvalid ? tri.light : kInvalid;
        if (light != kInvalid) light += in.light_offset;
        out.light = light;
    }
    out.position = o + d * t;
    return true;
}

}  // namespace wf
