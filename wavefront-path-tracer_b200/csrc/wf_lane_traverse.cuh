// Lane-refill traversal for the wavefront trace and shadow kernels.
//
// trace_closest / trace_any (wf_traverse.cuh) run one ray to completion per
// thread, so a warp lasts as long as its longest ray and most lanes sit idle
// behind a few grazing rays.  Here each lane's traversal is a resumable state
// machine (one node or one leaf per step) and lanes that finish take the next
// ray from the queue while the others keep going (the "replace terminated
// rays" scheme of Aila and Laine, "Understanding the Efficiency of Ray
// Traversal on GPUs", HPG 2009).
//
// Per ray nothing changes: the stages run in traceRay / isOccluded order
// (direct spheres, direct instances, static triangles, TLAS with instance
// BLASes, direct triangle BVH or list), every slab and triangle test has the
// same operands, the near-first child order and the popped-entry re-test
// "entry < closestT" are those of bvh_closest / tlas_closest, and the sphere
// bookkeeping follows instance_closest and trace_closest.  The TLAS path and
// the BLAS path below it share one stack: BLAS entries sit above the TLAS
// entries and the BLAS is finished when the stack drops back to its base.
#pragma once

#include "wf_traverse.cuh"

namespace wf {

// TLAS path + BLAS path, each at most kMaxBvhDepth (60) entries deep.
constexpr int kLaneStack = 128;

enum : uint32_t { kStageTlas = 0, kStageBlas = 1, kStageDirect = 2, kStageDone = 3 };

// The traversal stack keeps its most recent entry in registers (top_ref,
// top_t) and the entries below it in local memory, one 8-byte (ref, entry
// distance) pair each.  The usual pattern -- push the far child, descend
// the near one to a leaf, pop the far child -- then resumes from a register
// instead of waiting on a local-memory load; the refill of the register
// from memory is issued at the pop and is ready by the next one.
struct ClosestLane {
    V3 wo, wd;            // world ray
    V3 o, d, inv;         // ray of the current BVH (instance-local inside a BLAS)
    TraceState h;
    int ref;              // node (>= 0) or ~leaf to process next
    uint32_t stage;
    int size, base;       // stack size (the top included); first entry of the current BVH
    uint32_t inst, material_override;
    float previous;       // closestT when the current BLAS / direct BVH was entered
    int top_ref;          // entry size - 1 (valid when size > 0)
    float top_t;
    int2 stack[kLaneStack];  // entries 0 .. size - 2: (ref, entry distance bits)
};

WF_DEV void lane_push(ClosestLane& L, int ref, float t) {
    if (L.size >= kLaneStack) return;  // TLAS + BLAS depth <= 2 * kMaxBvhDepth < kLaneStack
    if (L.size > 0) L.stack[L.size - 1] = make_int2(L.top_ref, __float_as_int(L.top_t));
    L.top_ref = ref;
    L.top_t = t;
    ++L.size;
}

// Removes the top entry (size > 0) into (ref, t) and brings the next one
// into the registers.
WF_DEV void lane_pop(ClosestLane& L, int& ref, float& t) {
    ref = L.top_ref;
    t = L.top_t;
    --L.size;
    if (L.size > 0) {
        int2 e = L.stack[L.size - 1];
        L.top_ref = e.x;
        L.top_t = __int_as_float(e.y);
    }
}

// Direct triangle list (last stage of traceRay): its BVH is traversed by the
// lane; the no-BVH linear list runs at once.
template <typename Tally>
WF_DEV void closest_begin_direct(ClosestLane& L, const DeviceScene& s, Tally& tally) {
    L.stage = kStageDone;
    if (s.direct_count == 0) return;
    L.previous = L.h.t;
    if (s.direct_bvh.root != kNoRoot) {
        L.o = L.wo;
        L.d = L.wd;
        L.inv = inverse_direction(L.wd);
        float near_t;
        if (!slab_box(L.o, L.inv, s.direct_bvh.box, L.h.t, near_t)) return;
        L.stage = kStageDirect;
        L.size = L.base = 0;
        L.ref = s.direct_bvh.root;
        return;
    }
    TraceState& h = L.h;
    for (uint32_t i = 0; i < s.direct_count; ++i) {
        uint32_t ti = s.direct_first + i;
        tally.triangle();
        TriVerts tri = load_triangle(s, ti);
        float t, u, v;
        if (!intersect_triangle(L.wo, L.wd, tri.v0, tri.v1, tri.v2, t, u, v) || t >= h.t) continue;
        if (alpha_rejects<Tally>(s, tri.material, ti, u, v)) continue;
        h.t = t;
        h.u = u;
        h.v = v;
        h.prim = make_prim(kHitTriangle, ti);
        h.inst = kInvalid;
    }
    if (h.t < L.previous) h.sphere = kInvalid;
}

// Starts a ray: the linear stages of traceRay, then the TLAS root.
template <typename Tally>
WF_DEV void closest_begin(ClosestLane& L, const DeviceScene& s, V3 o, V3 d, Tally& tally) {
    TraceState& h = L.h;
    trace_state_init(h, 1e30f);
    L.wo = o;
    L.wd = d;
    for (uint32_t i = 0; i < s.direct_sphere_count; ++i) sphere_closest(s, s.direct_spheres[i], o, d, h, tally);
    for (uint32_t i = 0; i < s.direct_instance_count; ++i)
        instance_closest(s, s.direct_instances[i], o, d, h, false, tally);
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
    L.size = L.base = 0;
    if (s.tlas.root != kNoRoot) {
        L.o = o;
        L.d = d;
        L.inv = inverse_direction(d);
        float near_t;
        if (slab_box(o, L.inv, s.tlas.box, h.t, near_t)) {
            L.stage = kStageTlas;
            L.ref = s.tlas.root;
            return;
        }
    }
    closest_begin_direct(L, s, tally);
}

// Pops the next entry whose box still starts before closestT; finishes BVHs
// whose entries are exhausted (BLAS -> TLAS -> direct -> done).
template <typename Tally>
WF_DEV void closest_pop(ClosestLane& L, const DeviceScene& s, Tally& tally) {
    for (;;) {
        if (L.size == L.base) {
            if (L.stage == kStageBlas) {
                if (L.h.t < L.previous) L.h.sphere = kInvalid;
                L.stage = kStageTlas;
                L.base = 0;
                L.o = L.wo;
                L.d = L.wd;
                L.inv = inverse_direction(L.wd);
                continue;
            }
            if (L.stage == kStageTlas) {
                closest_begin_direct(L, s, tally);
                return;
            }
            if (L.h.t < L.previous) L.h.sphere = kInvalid;  // direct BVH finished
            L.stage = kStageDone;
            return;
        }
        int ref;
        float t;
        lane_pop(L, ref, t);
        if (t < L.h.t) {
            L.ref = ref;
            return;
        }
    }
}

// One node or one leaf of the current BVH.
template <typename Tally>
WF_DEV void closest_step(ClosestLane& L, const DeviceScene& s, Tally& tally) {
    int ref = L.ref;
    if (ref >= 0) {
        tally.node();
        const BvhNode* node = &s.nodes[ref];
        float4 lxy = __ldg(&node->lxy);
        float4 rxy = __ldg(&node->rxy);
        float4 lrz = __ldg(&node->lrz);
        int4 ch = __ldg(&node->child);
        float tl, tr;
        bool hl = slab(L.o, L.inv, lxy.x, lxy.y, lxy.z, lxy.w, lrz.x, lrz.y, L.h.t, tl);
        bool hr = slab(L.o, L.inv, rxy.x, rxy.y, rxy.z, rxy.w, lrz.z, lrz.w, L.h.t, tr);
        if (hl && hr) {
            bool left_near = tl < tr;
            lane_push(L, left_near ? ch.y : ch.x, left_near ? tr : tl);
            L.ref = left_near ? ch.x : ch.y;
            return;
        }
        if (hl) { L.ref = ch.x; return; }
        if (hr) { L.ref = ch.y; return; }
    } else if (L.stage == kStageTlas) {
        uint32_t leaf = __ldg(&s.tlas_leaves[~ref]);
        if (leaf & 0x80000000u) {
            sphere_closest(s, leaf & 0x7fffffffu, L.o, L.d, L.h, tally);
        } else {
            // intersectMeshInstance with useBvh = true (device_traversal.cuh:802-834)
            tally.instance();
            Instance in = load_instance(s, leaf);
            Blas b = s.blases[in.blas];
            V3 lo = to_local_vector(in, L.wo - instance_translation(in));
            V3 ld = to_local_vector(in, L.wd);
            L.previous = L.h.t;
            if (b.bvh.root != kNoRoot) {
                V3 linv = inverse_direction(ld);
                float near_t;
                if (slab_box(lo, linv, b.bvh.box, L.h.t, near_t)) {
                    L.o = lo;
                    L.d = ld;
                    L.inv = linv;
                    L.inst = leaf;
                    L.material_override = in.material_override;
                    L.stage = kStageBlas;
                    L.base = L.size;
                    L.ref = b.bvh.root;
                    return;
                }
            } else {
                mesh_linear_closest(s, b, lo, ld, L.h, leaf, in.material_override, tally);
                if (L.h.t < L.previous) L.h.sphere = kInvalid;
            }
        }
    } else {
        bool blas = L.stage == kStageBlas;
        uint32_t ti = uint32_t(~ref);
        tally.triangle();
        TriVerts tri = load_triangle(s, ti);
        float t, u, v;
        if (intersect_triangle(L.o, L.d, tri.v0, tri.v1, tri.v2, t, u, v) && t < L.h.t) {
            uint32_t override_m = blas ? L.material_override : kInvalid;
            uint32_t m = override_m == kInvalid ? tri.material : override_m;
            if (!alpha_rejects<Tally>(s, m, ti, u, v)) {
                L.h.t = t;
                L.h.u = u;
                L.h.v = v;
                L.h.prim = make_prim(blas ? kHitMesh : kHitTriangle, ti);
                L.h.inst = blas ? L.inst : kInvalid;
            }
        }
    }
    closest_pop(L, s, tally);
}

struct AnyLane {
    V3 wo, wd;
    V3 o, d, inv;
    float t_max;
    int ref;
    uint32_t stage;
    int size, base;
    uint32_t material_override;
    bool hit;
    int stack_ref[kLaneStack];
};

template <typename Tally>
WF_DEV void any_begin_direct(AnyLane& L, const DeviceScene& s, Tally& tally) {
    L.stage = kStageDone;
    if (s.direct_count == 0) return;
    if (s.direct_bvh.root != kNoRoot) {
        L.o = L.wo;
        L.d = L.wd;
        L.inv = inverse_direction(L.wd);
        float near_t;
        if (!slab_box(L.o, L.inv, s.direct_bvh.box, L.t_max, near_t)) return;
        L.stage = kStageDirect;
        L.size = L.base = 0;
        L.ref = s.direct_bvh.root;
        return;
    }
    for (uint32_t i = 0; i < s.direct_count; ++i) {
        tally.triangle();
        TriVerts tri = load_triangle(s, s.direct_first + i);
        float t, u, v;
        if (intersect_triangle(L.wo, L.wd, tri.v0, tri.v1, tri.v2, t, u, v) && t < L.t_max &&
            !alpha_rejects<Tally>(s, tri.material, s.direct_first + i, u, v)) {
            L.hit = true;
            return;
        }
    }
}

// Starts an occlusion ray: the linear stages of isOccluded, then the TLAS root.
template <typename Tally>
WF_DEV void any_begin(AnyLane& L, const DeviceScene& s, V3 o, V3 d, float t_max, Tally& tally) {
    L.wo = o;
    L.wd = d;
    L.t_max = t_max;
    L.hit = false;
    L.stage = kStageDone;
    for (uint32_t i = 0; i < s.direct_sphere_count; ++i) {
        float t;
        tally.sphere();
        if (intersect_sphere(o, d, __ldg(&s.spheres[s.direct_spheres[i]]), t) && t < t_max) {
            L.hit = true;
            return;
        }
    }
    for (uint32_t i = 0; i < s.direct_instance_count; ++i)
        if (instance_any(s, s.direct_instances[i], o, d, t_max, false, tally)) {
            L.hit = true;
            return;
        }
    for (uint32_t i = 0; i < s.static_count; ++i) {
        tally.triangle();
        TriVerts tri = load_triangle(s, s.static_first + i);
        float t, u, v;
        if (intersect_triangle(o, d, tri.v0, tri.v1, tri.v2, t, u, v) && t < t_max &&
            !alpha_rejects<Tally>(s, tri.material, s.static_first + i, u, v)) {
            L.hit = true;
            return;
        }
    }
    L.size = L.base = 0;
    if (s.tlas.root != kNoRoot) {
        L.o = o;
        L.d = d;
        L.inv = inverse_direction(d);
        float near_t;
        if (slab_box(o, L.inv, s.tlas.box, t_max, near_t)) {
            L.stage = kStageTlas;
            L.ref = s.tlas.root;
            return;
        }
    }
    any_begin_direct(L, s, tally);
}

template <typename Tally>
WF_DEV void any_pop(AnyLane& L, const DeviceScene& s, Tally& tally) {
    for (;;) {
        if (L.size == L.base) {
            if (L.stage == kStageBlas) {
                L.stage = kStageTlas;
                L.base = 0;
                L.o = L.wo;
                L.d = L.wd;
                L.inv = inverse_direction(L.wd);
                continue;
            }
            if (L.stage == kStageTlas) {
                any_begin_direct(L, s, tally);
                return;
            }
            L.stage = kStageDone;
            return;
        }
        L.ref = L.stack_ref[--L.size];
        return;
    }
}

template <typename Tally>
WF_DEV void any_step(AnyLane& L, const DeviceScene& s, Tally& tally) {
    int ref = L.ref;
    if (ref >= 0) {
        tally.node();
        const BvhNode* node = &s.nodes[ref];
        float4 lxy = __ldg(&node->lxy);
        float4 rxy = __ldg(&node->rxy);
        float4 lrz = __ldg(&node->lrz);
        int4 ch = __ldg(&node->child);
        float tl, tr;
        bool hl = slab(L.o, L.inv, lxy.x, lxy.y, lxy.z, lxy.w, lrz.x, lrz.y, L.t_max, tl);
        bool hr = slab(L.o, L.inv, rxy.x, rxy.y, rxy.z, rxy.w, lrz.z, lrz.w, L.t_max, tr);
        if (hl && hr) {
            bool left_near = tl < tr;
            if (L.size < kLaneStack) L.stack_ref[L.size++] = left_near ? ch.y : ch.x;
            L.ref = left_near ? ch.x : ch.y;
            return;
        }
        if (hl) { L.ref = ch.x; return; }
        if (hr) { L.ref = ch.y; return; }
    } else if (L.stage == kStageTlas) {
        uint32_t leaf = __ldg(&s.tlas_leaves[~ref]);
        if (leaf & 0x80000000u) {
            float t;
            tally.sphere();
            if (intersect_sphere(L.o, L.d, __ldg(&s.spheres[leaf & 0x7fffffffu]), t) && t < L.t_max) {
                L.hit = true;
                L.stage = kStageDone;
                return;
            }
        } else {
            tally.instance();
            Instance in = load_instance(s, leaf);
            Blas b = s.blases[in.blas];
            V3 lo = to_local_vector(in, L.wo - instance_translation(in));
            V3 ld = to_local_vector(in, L.wd);
            if (b.bvh.root != kNoRoot) {
                V3 linv = inverse_direction(ld);
                float near_t;
                if (slab_box(lo, linv, b.bvh.box, L.t_max, near_t)) {
                    L.o = lo;
                    L.d = ld;
                    L.inv = linv;
                    L.material_override = in.material_override;
                    L.stage = kStageBlas;
                    L.base = L.size;
                    L.ref = b.bvh.root;
                    return;
                }
            } else {
                for (uint32_t i = 0; i < b.count; ++i) {
                    tally.triangle();
                    TriVerts tri = load_triangle(s, s.mesh_linear[b.first_linear + i]);
                    float t, u, v;
                    if (!intersect_triangle(lo, ld, tri.v0, tri.v1, tri.v2, t, u, v) || t >= L.t_max) continue;
                    uint32_t m = in.material_override == kInvalid ? tri.material : in.material_override;
                    if (!alpha_rejects<Tally>(s, m, s.mesh_linear[b.first_linear + i], u, v)) {
                        L.hit = true;
                        L.stage = kStageDone;
                        return;
                    }
                }
            }
        }
    } else {
        uint32_t ti = uint32_t(~ref);
        tally.triangle();
        TriVerts tri = load_triangle(s, ti);
        float t, u, v;
        if (intersect_triangle(L.o, L.d, tri.v0, tri.v1, tri.v2, t, u, v) && t < L.t_max) {
            uint32_t override_m = L.stage == kStageBlas ? L.material_override : kInvalid;
            uint32_t m = override_m == kInvalid ? tri.material : override_m;
            if (!alpha_rejects<Tally>(s, m, ti, u, v)) {
                L.hit = true;
                L.stage = kStageDone;
                return;
            }
        }
    }
    any_pop(L, s, tally);
}

// Lane refill: when at least `threshold` lanes of the warp are idle (or all
// of them), the idle lanes take the next rays of [0, n) from `counter` with
// one warp-aggregated atomic.  Returns the ray index for this lane, or
// kInvalid.  `more` (warp-uniform) turns false once the counter passes n.
WF_DEV uint32_t refill(uint32_t* counter, uint32_t n, bool idle, uint32_t threshold, bool& more) {
    unsigned mask = __ballot_sync(0xffffffffu, idle);
    if (!more || mask == 0) return kInvalid;
    uint32_t k = __popc(mask);
    if (k < threshold && mask != 0xffffffffu) return kInvalid;
    uint32_t lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, k);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base + k >= n) more = false;
    if (!idle) return kInvalid;
    uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
    return slot < n ? slot : kInvalid;
}

}  // namespace wf
