// Wavefront kernels and the render loop.
//
// Graph mode (replaces RenderDriver::createWavefrontGraph,
// src/renderer/render_driver.cu:264-297): per tile-sample the stream replays
//   raygen, maxDepth x { trace, shade, shadow, finalize }, advance
// captured once as a CUDA graph.  trace = closest hit of every queued path
// (lean traversal kernel); shade = material/NEE evaluation that queues shadow
// rays instead of tracing them inline; shadow = any-hit over the compacted
// shadow queue; finalize = ordered radiance accumulation, framebuffer writes
// of finished paths and warp-ballot compaction of survivors (the reference's
// appendWarpCompacted, include/renderer/queue_compaction.cuh:8-29).
//
// Persistent mode (replaces persistentWavefrontTrace, renderer.cu:55-125): one
// cooperative launch per tile-sample; warps pull 32-path chunks from a
// per-bounce work counter, trace + shade + shadow inline, compact, and meet at
// a bounded grid barrier between bounces.
#include "wf_renderer.h"
#include "wf_shade.cuh"
#include "wf_lane_traverse.cuh"
#include "wf_wavefront.cuh"

#include <cuda.h>

#include <algorithm>
#include <cstring>
#include <type_traits>

namespace wf {

wf_status cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? WF_ERR_OOM : WF_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define WF_CUDA(call)                                          \
    do {                                                       \
        cudaError_t wf_e_ = (call);                            \
        if (wf_e_ != cudaSuccess) return cuda_fail(wf_e_, #call); \
    } while (0)

namespace {

// Camera rays of tile.samples samples (graph mode's wave; 1 elsewhere):
// slot k * P + q is pixel q of the tile in sample sample_index + k, so each
// sample's rays sit together in pixel order.
WF_DEV void raygen_stage(RenderParams rp, const TileDev* tile_ptr, Counters* c, PathSoA ps, uint32_t* queue, uint32_t capacity) {
    TileDev tile = *tile_ptr;
    uint32_t pixels = tile.width * tile.height;
    uint32_t n = uint32_t(min(uint64_t(pixels) * tile.samples, uint64_t(capacity)));
    uint32_t sample = c->sample_index;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        c->queue_count[0] = n;
        c->paths += n;
        c->work_trace = 0;
    }
    for (uint32_t lp = gid; lp < n; lp += gridDim.x * blockDim.x) {
        uint32_t k = lp / pixels;
        Path path;
        init_path(rp, tile, sample + k, lp - k * pixels, path);
        store_path(ps, lp, path);
        ps.radiance[lp] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        queue[lp] = lp;
    }
}

__global__ void k_raygen(RenderParams rp, const TileDev* tile_ptr, Counters* c, PathSoA ps, uint32_t* queue,
                         uint32_t capacity) {
    count_launch(c);
    raygen_stage(rp, tile_ptr, c, ps, queue, capacity);
}

// Streaming mode: every slot (= pixel of the tile) starts the launch's first
// sample; slot_sample counts the samples a slot has started.
__global__ void k_raygen_stream(RenderParams rp, const TileDev* tile_ptr, Counters* c, PathSoA ps, uint32_t* queue,
                                uint32_t capacity) {
    count_launch(c);
    TileDev tile = *tile_ptr;
    uint32_t n = min(tile.width * tile.height, capacity);
    uint32_t sample = c->sample_index;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        // every slot starts with a camera ray: queue 0 holds no survivors yet
        c->queue_count[0] = 0;
        c->camera_count[0] = n;
        c->camera_count[1] = 0;
        c->paths += uint64_t(n) * tile.samples;
        c->work_trace = 0;
        c->work_camera = 0;
        c->stream_iterations = 0;
    }
    for (uint32_t lp = gid; lp < n; lp += gridDim.x * blockDim.x) {
        Path path;
        init_path(rp, tile, sample, lp, path);
        store_path(ps, lp, path);
        ps.radiance[lp] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.slot_sample[lp] = 0;
        ps.wait[lp] = 0;
        queue[lp] = lp;
    }
}

// kLanes: lane-refill state machines (incoherent bounces).  Otherwise each
// warp takes 32 consecutive queue entries and every lane runs its ray to the
// end (camera rays: neighbouring pixels visit the same nodes in lockstep).
// The per-ray visit order and arithmetic are the same either way.
// The closest-hit stage of one bounce; the kernels below differ only in
// their register bounds.
// `camera` (nullable, streaming mode): the number of camera rays of slots
// that started a sample, queued after the *count survivors.  Two launches
// share the bounce: when survivors exist, the lane-refill launch traces them
// and the camera rays behind them (a warp that holds a long survivor keeps
// refilling its other lanes with camera rays, which sit in runs of
// neighbouring pixels), and the per-thread launch (kLanes false) has nothing
// to do; when no path survived (the first pass, or a drained queue) the
// per-thread launch traces the camera rays alone, taking its work from
// `work`.  The lane-refill launch makes the per-bounce resets.
template <typename Tally, bool kLanes>
WF_DEV void trace_stage(const DeviceScene& s, PathSoA ps, const uint32_t* queue, const uint32_t* count, float4* hit_a,
                        uint32_t* hit_inst, Counters* c, uint32_t bounce, TallyTotals* totals, uint32_t refill_at,
                        const uint32_t* camera, uint32_t* work) {
    count_launch(c);
    uint32_t n = *count;
    uint32_t* counter = &c->work_trace;
    bool resets = true;
    if (camera) {
        uint32_t survivors = n, rays = *camera;
        if constexpr (kLanes) {
            n = survivors ? survivors + rays : 0u;
        } else {
            n = survivors ? 0u : rays;
            counter = work;
            resets = false;
        }
    }
    constexpr uint32_t first = 0;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        if (resets) {
            c->shadow_count = 0;
            c->gather_count = 0;
            c->dense_count = 0;
            c->work_shade = 0;
            for (int k = 0; k < 8; ++k) c->shade_bucket[k] = c->shade_cursor[k] = 0;
            if (bounce < kMaxBounces) c->profile[bounce] = n;
        }
        atomicAdd(&c->extension_rays, (unsigned long long)n);
    }
    Tally tally;
    if constexpr (!kLanes) {
        uint32_t base;
        while (next_chunk(counter, n, base)) {
            uint32_t i = first + base + (threadIdx.x & 31);
            if (i >= first + n) continue;
            uint32_t p = queue[i];
            float4 o = ps.origin[p], d = ps.direction[p];
            TraceState h;
            trace_closest(s, f4xyz(o), f4xyz(d), h, tally);
            hit_a[i] = make_float4(h.t, h.u, h.v, __uint_as_float(h.prim));
            hit_inst[i] = h.inst;
        }
        if constexpr (Tally::kCounts) flush_tally(tally, totals);
        return;
    }
    ClosestLane L;
    L.stage = kStageDone;
    uint32_t i = 0;
    bool more = true;
    for (;;) {
        bool idle = L.stage == kStageDone;
        uint32_t slot = refill(counter, n, idle, refill_at, more);
        if (slot != kInvalid) {
            i = first + slot;
            uint32_t p = queue[i];
            float4 o = ps.origin[p], d = ps.direction[p];
            closest_begin(L, s, f4xyz(o), f4xyz(d), tally);
            if (L.stage == kStageDone) {
                hit_a[i] = make_float4(L.h.t, L.h.u, L.h.v, __uint_as_float(L.h.prim));
                hit_inst[i] = L.h.inst;
            }
        }
        bool busy = L.stage != kStageDone;
        if (!__any_sync(0xffffffffu, busy)) {
            if (!more) break;
            continue;
        }
        if (busy) {
            closest_step(L, s, tally);
            if (L.stage == kStageDone) {
                hit_a[i] = make_float4(L.h.t, L.h.u, L.h.v, __uint_as_float(L.h.prim));
                hit_inst[i] = L.h.inst;
            }
        }
    }
    if constexpr (Tally::kCounts) flush_tally(tally, totals);
}

// Lane-refill bounces: at most 72 registers (7 CTAs of 128 per SM): 8 bytes
// of spill cost less than the warps a 79-register allocation (6 CTAs) leaves
// out; a 64-register cap spills far more.  __maxnreg__ keeps every block
// size launchable.
template <typename Tally, bool kLanes = true>
__global__ void __maxnreg__(72) k_trace(DeviceScene s, PathSoA ps, const uint32_t* queue, const uint32_t* count,
                                        float4* hit_a, uint32_t* hit_inst, Counters* c, uint32_t bounce,
                                        TallyTotals* totals, uint32_t refill_at, const uint32_t* camera,
                                        uint32_t* work) {
    trace_stage<Tally, kLanes>(s, ps, queue, count, hit_a, hit_inst, c, bounce, totals, refill_at, camera, work);
}

// Camera rays (one traversal per thread, coherent): bounded to 8 CTAs of 128
// per SM (64 registers).  Unlike the lane-refill loop, this traversal gains
// more from the extra warps than its spills cost: bounce 0 of the 1080p large
// mesh 2.07 -> 1.98 ms, the frame +0.6 %.
template <typename Tally>
__global__ void __launch_bounds__(128, 8) k_trace_camera(DeviceScene s, PathSoA ps, const uint32_t* queue,
                                                         const uint32_t* count, float4* hit_a, uint32_t* hit_inst,
                                                         Counters* c, uint32_t bounce, TallyTotals* totals,
                                                         uint32_t refill_at, const uint32_t* camera, uint32_t* work) {
    trace_stage<Tally, false>(s, ps, queue, count, hit_a, hit_inst, c, bounce, totals, refill_at, camera, work);
}

// Shading categories: warps of k_shade take entries of one category at a
// time, so they run one material branch instead of all of them.  Which warp
// shades which path does not change any path's arithmetic: the outputs go to
// the entry's own queue position.
WF_DEV uint32_t shade_category(const DeviceScene& s, float4 ha, uint32_t inst) {
    uint32_t prim = __float_as_uint(ha.w);
    uint32_t kind = hit_kind(prim), index = hit_index(prim);
    if (kind == kHitMiss) return 0;
    uint32_t m;
    if (kind == kHitSphere) {
        m = s.sphere_materials[index];
    } else {
        m = __float_as_uint(__ldg(&s.triangles[3 * size_t(index) + 1]).w);
        if (kind == kHitMesh) {
            uint32_t over = load_instance(s, inst).material_override;
            if (over != kInvalid) m = over;
        }
    }
    return material_category(s.materials[m]);
}

WF_DEV void classify_stage(const DeviceScene& s, const uint32_t* count, const float4* hit_a, const uint32_t* hit_inst, uint8_t* key, Counters* c) {
    __shared__ uint32_t histogram[kShadeCategories];
    if (threadIdx.x < kShadeCategories) histogram[threadIdx.x] = 0;
    __syncthreads();
    uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k = shade_category(s, hit_a[i], hit_inst[i]);
        key[i] = uint8_t(k);
        atomicAdd(&histogram[k], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kShadeCategories && histogram[threadIdx.x])
        atomicAdd(&c->shade_bucket[threadIdx.x], histogram[threadIdx.x]);
}

__global__ void k_classify(const __grid_constant__ DeviceScene s, const uint32_t* count, const float4* hit_a,
                           const uint32_t* hit_inst, uint8_t* key, Counters* c) {
    count_launch(c);
    classify_stage(s, count, hit_a, hit_inst, key, c);
}

// Counting-sort scatter: within a warp, entries of one category keep their
// order (ballot rank); warps reserve runs of each bucket with one atomic.
WF_DEV void scatter_stage(const uint32_t* count, const uint8_t* key, uint32_t* order, Counters* c) {
    uint32_t n = *count;
    uint32_t offset[kShadeCategories];
    uint32_t run = 0;
    for (uint32_t k = 0; k < kShadeCategories; ++k) {
        offset[k] = run;
        run += c->shade_bucket[k];
    }
    uint32_t lane = threadIdx.x & 31;
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = warp * 32; base < n; base += warps * 32) {
        uint32_t i = base + lane;
        uint32_t k = i < n ? key[i] : kShadeCategories;
        unsigned peers = __match_any_sync(0xffffffffu, k);
        uint32_t leader = __ffs(peers) - 1;
        uint32_t start = 0;
        if (lane == leader && k < kShadeCategories) start = atomicAdd(&c->shade_cursor[k], uint32_t(__popc(peers)));
        start = __shfl_sync(0xffffffffu, start, leader);
        if (k < kShadeCategories) order[offset[k] + start + __popc(peers & ((1u << lane) - 1u))] = i;
    }
}

__global__ void k_scatter(const uint32_t* count, const uint8_t* key, uint32_t* order, Counters* c) {
    count_launch(c);
    scatter_stage(count, key, order, c);
}

// 128 registers: 4 CTAs per SM; the few spills cost less than the lost warps.
template <bool kTextures>
WF_DEV void shade_stage(const DeviceScene& s, const RenderParams& rp, PathSoA ps, const uint32_t* queue, const uint32_t* count, const float4* hit_a, const uint32_t* hit_inst, float4* terms, int4* shade_out, float4* shadow_origin, float4* shadow_dir, uint32_t shadow_capacity, Counters* c, uint32_t* next_count, GatherQueue gathers, const uint32_t* order) {
    uint32_t n = *count;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        *next_count = 0;
        c->work_shadow = 0;
        c->work_gather = 0;
        c->work_dense = 0;
    }
    uint32_t base;
    while (next_chunk(&c->work_shade, n, base)) {
        uint32_t j = base + (threadIdx.x & 31);
        if (j >= n) continue;
        uint32_t i = order ? order[j] : j;
        uint32_t p = queue[i];
        Path path = load_path(ps, p);
        float4 ha = hit_a[i];
        SurfaceHit sh;
        bool did_hit = finish_hit(s, path.origin, path.direction, ha.x, ha.y, ha.z, __float_as_uint(ha.w),
                                  hit_inst[i], sh);
        DeferredSink sink;
        sink.shadow_origin = shadow_origin;
        sink.shadow_dir = shadow_dir;
        sink.shadow_count = &c->shadow_count;
        sink.shadow_capacity = shadow_capacity;
        sink.terms = terms + size_t(i) * kMaxTerms;
        sink.owner = i;
        sink.tag = i;
        sink.nterms = 0;
        sink.kill = kUnconditional;
        sink.overflow = &c->overflow;
        sink.gathers = gathers;
        bool alive = shade_path<DeferredSink, kTextures>(s, rp, path, did_hit, sh, sink);
        if (sink.nterms > kMaxTerms) atomicOr(&c->overflow, 2u);
        store_path(ps, p, path);
        shade_out[i] = make_int4(min(sink.nterms, kMaxTerms), sink.kill, alive ? 1 : 0, 0);
    }
}

template <bool kTextures>
__global__ void __launch_bounds__(128, 4) k_shade(const __grid_constant__ DeviceScene s, const __grid_constant__ RenderParams rp, PathSoA ps, const uint32_t* queue, const uint32_t* count,
                        const float4* hit_a, const uint32_t* hit_inst, float4* terms, int4* shade_out,
                        float4* shadow_origin, float4* shadow_dir, uint32_t shadow_capacity, Counters* c,
                        uint32_t* next_count, GatherQueue gathers, const uint32_t* order) {
    count_launch(c);
    shade_stage<kTextures>(s, rp, ps, queue, count, hit_a, hit_inst, terms, shade_out, shadow_origin, shadow_dir, shadow_capacity, c, next_count, gathers, order);
}

// Caustic gathers queued by k_shade (gatherCaustics, photon_mapping.cu:91-163),
// written into the term slots their paths reserved.  A request whose cells
// hold many photons (near a caustic) would scan them serially while the rest
// of the GPU waits; it goes to k_gather_dense, one warp per request.
constexpr uint32_t kDenseGather = 256;

WF_DEV void write_gather_term(const RenderParams& rp, const GatherQueue& q, float4* terms, uint32_t r, V3 caustic) {
    float4 pos = q.position[r], nrm = q.normal[r], thr = q.throughput[r], alb = q.albedo[r];
    Path depth_only{};
    depth_only.depth = nrm.w != 0.0f ? 1u : 0u;
    V3 col = clamp_contribution(depth_only, hadamard(f4xyz(thr), hadamard(f4xyz(alb), caustic)), rp.clamp, false);
    terms[__float_as_uint(pos.w)] = make_float4(col.x, col.y, col.z, __int_as_float(kUnconditional));
}

WF_DEV void gather_stage(const RenderParams& rp, GatherQueue q, float4* terms, Counters* c) {
    uint32_t n = min(*q.count, q.capacity);
    uint32_t base;
    while (next_chunk(&c->work_gather, n, base)) {
        uint32_t r = base + (threadIdx.x & 31);
        if (r >= n) continue;
        float4 pos = q.position[r], nrm = q.normal[r];
        if (gather_cell_photons(rp.photons, f4xyz(pos), rp.gather_radius) > kDenseGather) {
            q.dense[atomicAdd(q.dense_count, 1u)] = r;
            continue;
        }
        ShadeHit hit{};
        hit.position = f4xyz(pos);
        hit.normal = f4xyz(nrm);
        write_gather_term(rp, q, terms, r, gather_caustics(rp.photons, hit, rp.gather_radius));
    }
}

__global__ void k_gather(const __grid_constant__ RenderParams rp, GatherQueue q, float4* terms, Counters* c) {
    count_launch(c);
    gather_stage(rp, q, terms, c);
}

WF_DEV void gather_dense_stage(const RenderParams& rp, GatherQueue q, float4* terms, Counters* c) {
    uint32_t n = min(*q.dense_count, q.capacity);
    uint32_t lane = threadIdx.x & 31;
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(&c->work_dense, 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= n) break;
        uint32_t r = q.dense[k];
        float4 pos = q.position[r], nrm = q.normal[r];
        V3 caustic = gather_caustics_warp(rp.photons, f4xyz(pos), f4xyz(nrm), rp.gather_radius);
        if (lane == 0) write_gather_term(rp, q, terms, r, caustic);
    }
}

__global__ void k_gather_dense(const __grid_constant__ RenderParams rp, GatherQueue q, float4* terms, Counters* c) {
    count_launch(c);
    gather_dense_stage(rp, q, terms, c);
}

template <typename Tally>
WF_DEV void shadow_stage(DeviceScene s, const float4* shadow_origin, const float4* shadow_dir, uint8_t* result, Counters* c, uint32_t capacity, TallyTotals* totals, uint32_t refill_at) {
    uint32_t n = min(c->shadow_count, capacity);
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) c->shadow_rays += n;
    Tally tally;
    AnyLane L;
    L.stage = kStageDone;
    uint32_t j = 0;
    bool more = true;
    for (;;) {
        bool idle = L.stage == kStageDone;
        uint32_t slot = refill(&c->work_shadow, n, idle, refill_at, more);
        if (slot != kInvalid) {
            j = slot;
            float4 o = shadow_origin[j], d = shadow_dir[j];
            any_begin(L, s, f4xyz(o), f4xyz(d), o.w, tally);
            if (L.stage == kStageDone) result[j] = L.hit ? 1 : 0;
        }
        bool busy = L.stage != kStageDone;
        if (!__any_sync(0xffffffffu, busy)) {
            if (!more) break;
            continue;
        }
        if (busy) {
            any_step(L, s, tally);
            if (L.stage == kStageDone) result[j] = L.hit ? 1 : 0;
        }
    }
    if constexpr (Tally::kCounts) flush_tally(tally, totals);
}

template <typename Tally>
__global__ void k_shadow(DeviceScene s, const float4* shadow_origin, const float4* shadow_dir, uint8_t* result,
                         Counters* c, uint32_t capacity, TallyTotals* totals, uint32_t refill_at) {
    count_launch(c);
    shadow_stage<Tally>(s, shadow_origin, shadow_dir, result, c, capacity, totals, refill_at);
}

// Adds each path's accepted terms in emission order, applies the kill rule,
// adds ended paths to the framebuffer and compacts survivors into `next`
// (appendWarpCompacted, queue_compaction.cuh:8-29).  With kRegenerate (the
// streaming mode) an ended path's slot is marked to start its pixel's next
// sample (k_regenerate); the framebuffer add comes first, so every pixel
// still accumulates its samples in sample order.
template <bool kRegenerate>
WF_DEV void finalize_stage(PathSoA ps, const uint32_t* queue, const uint32_t* count, const float4* terms, const int4* shade_out, const uint8_t* shadow_result, uint32_t* next, uint32_t* next_count, uint32_t capacity, float* framebuffer, uint32_t* work_trace, RenderParams rp, const TileDev* tile_ptr, Counters* c) {
    uint32_t n = *count;
    uint32_t lane = threadIdx.x & 31;
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) *work_trace = 0;
    for (uint32_t base = warp * 32; base < n; base += warps * 32) {
        uint32_t i = base + lane;
        bool alive = false;
        uint32_t p = 0;
        if (i < n) {
            p = queue[i];
            int4 so = shade_out[i];
            float4 r = ps.radiance[p];
            V3 rad = f4xyz(r);
            for (int k = 0; k < so.x; ++k) {
                float4 t = terms[size_t(i) * kMaxTerms + k];
                int h = __float_as_int(t.w);
                if (h < 0 || !shadow_result[h]) rad += f4xyz(t);
            }
            alive = so.z != 0 && !(so.y >= 0 && !shadow_result[so.y]);
            if (alive) {
                ps.radiance[p] = make_float4(rad.x, rad.y, rad.z, 0.0f);
            } else if (!kRegenerate && tile_ptr->samples > 1) {
                // a wave of several samples: k_accumulate_wave adds the
                // finished paths per pixel in sample order after the wave
                ps.radiance[p] = make_float4(rad.x, rad.y, rad.z, 1.0f);
            } else {
                uint32_t pixel = ps.info[p].x;
                float* f = framebuffer + 3 * size_t(pixel);
                f[0] += rad.x;
                f[1] += rad.y;
                f[2] += rad.z;
                if constexpr (kRegenerate) {
                    // the slot's next sample starts in k_regenerate
                    if (ps.slot_sample[p] + 1 < tile_ptr->samples) ps.wait[p] = 1;
                }
            }
        }
        unsigned mask = __ballot_sync(0xffffffffu, alive);
        uint32_t out = 0;
        if (lane == 0 && mask) out = atomicAdd(next_count, uint32_t(__popc(mask)));
        out = __shfl_sync(0xffffffffu, out, 0);
        uint32_t rank = __popc(mask & ((1u << lane) - 1u));
        if (alive && out + rank < capacity) next[out + rank] = p;
    }
}

// After a wave of several samples (graph mode): each pixel adds the
// radiance of its finished paths in sample order, the order in which
// one-sample launches would have added them, so the sums are the same.
__global__ void k_accumulate_wave(PathSoA ps, const TileDev* tile_ptr, float* framebuffer, Counters* c) {
    count_launch(c);
    TileDev tile = *tile_ptr;
    if (tile.samples <= 1) return;
    uint32_t pixels = tile.width * tile.height;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < pixels; q += gridDim.x * blockDim.x) {
        float* f = framebuffer + 3 * size_t(ps.info[q].x);
        float r = f[0], g = f[1], b = f[2];
        for (uint32_t k = 0; k < tile.samples; ++k) {
            float4 rad = ps.radiance[size_t(k) * pixels + q];
            if (rad.w != 0.0f) {
                r += rad.x;
                g += rad.y;
                b += rad.z;
            }
        }
        f[0] = r;
        f[1] = g;
        f[2] = b;
    }
}

template <bool kRegenerate>
__global__ void k_finalize(PathSoA ps, const uint32_t* queue, const uint32_t* count, const float4* terms,
                           const int4* shade_out, const uint8_t* shadow_result, uint32_t* next, uint32_t* next_count,
                           uint32_t capacity, float* framebuffer, uint32_t* work_trace, RenderParams rp,
                           const TileDev* tile_ptr, Counters* c) {
    count_launch(c);
    finalize_stage<kRegenerate>(ps, queue, count, terms, shade_out, shadow_result, next, next_count, capacity, framebuffer, work_trace, rp, tile_ptr, c);
}

// Streaming loop condition: run the body again while paths remain.  Each
// body pass advances every live path by two bounces.  A slot's path takes at
// most max_depth bounces, and a slot waits at most max_depth bounces for its
// next sample (within that many bounces every path in flight has ended, and
// an empty queue always regenerates), so a slot finishes within
// samples * 2 * max_depth bounces; a loop that exceeds that bound records an
// error and stops instead of spinning.
__global__ void k_stream_condition(cudaGraphConditionalHandle handle, Counters* c, const TileDev* tile,
                                   uint32_t max_depth) {
    count_launch(c);
    uint32_t it = ++c->stream_iterations;
    bool live = c->queue_count[0] + c->camera_count[0] > 0;
    uint64_t bound = uint64_t(tile->samples) * max_depth + 2;
    if (c->stream_limit && c->stream_limit < bound) bound = c->stream_limit;
    if (live && it >= bound) {
        c->error = kErrorStreamBound;
        live = false;
    }
    cudaGraphSetConditional(handle, live ? 1u : 0u);
}

__global__ void k_advance(Counters* c, const TileDev* tile) {
    count_launch(c);
    if (tile->advance_sample) c->sample_index += tile->samples;
}

// Streaming mode: once fewer than `percent` % of the tile's slots carry a
// path (or none does), every slot whose path ended and whose pixel has
// samples left starts its next sample.  Warps take 32 consecutive slots and
// append theirs with one atomic, so the camera rays queue after the
// survivors in runs of neighbouring pixels, which k_trace_camera traces
// coherently.  Per pixel the samples still run one after another.
__global__ void k_regenerate(const __grid_constant__ RenderParams rp, const TileDev* tile_ptr, Counters* c,
                             PathSoA ps, uint32_t* next, const uint32_t* next_count, uint32_t* camera_count,
                             uint32_t capacity, uint32_t percent) {
    count_launch(c);
    TileDev tile = *tile_ptr;
    uint32_t n = min(tile.width * tile.height, capacity);
    uint32_t alive = *next_count;
    if (alive != 0 && uint64_t(alive) * 100 >= uint64_t(n) * percent) return;
    uint32_t lane = threadIdx.x & 31;
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t sample = c->sample_index;
    for (uint32_t base = warp * 32; base < n; base += warps * 32) {
        uint32_t p = base + lane;
        bool waiting = p < n && ps.wait[p];
        unsigned mask = __ballot_sync(0xffffffffu, waiting);
        if (!mask) continue;
        uint32_t out = 0;
        if (lane == 0) out = atomicAdd(camera_count, uint32_t(__popc(mask)));
        out = __shfl_sync(0xffffffffu, out, 0);
        if (!waiting) continue;
        uint32_t started = ps.slot_sample[p] + 1;
        Path path;
        init_path(rp, tile, sample + started, p, path);
        store_path(ps, p, path);
        ps.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.slot_sample[p] = started;
        ps.wait[p] = 0;
        next[alive + out + __popc(mask & ((1u << lane) - 1u))] = p;
    }
}

// Streaming mode, after both traces of a bounce: the camera rays join the
// survivors, and their work counter is ready for the next bounce.
__global__ void k_merge_camera(Counters* c, uint32_t q) {
    count_launch(c);
    c->queue_count[q] += c->camera_count[q];
    c->camera_count[q] = 0;
    c->work_camera = 0;
}

// Grid barrier with a bounded wait.  All blocks are co-resident (cooperative
// launch).  A wait that exceeds ~2^31 cycles (or the watchdog's bound)
// records an error and gives up; callers then return and the host reports
// WF_ERR_TIMEOUT.
WF_DEV bool grid_barrier(Counters* c, uint32_t blocks) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t* gen = &c->barrier_generation;
        uint32_t g = *gen;
        long long limit = c->barrier_limit ? (long long)min(c->barrier_limit, 1ull << 62) : (1ll << 31);
        __threadfence();
        uint32_t arrived = atomicAdd(&c->barrier_count, 1u);
        if (arrived == blocks - 1) {
            c->barrier_count = 0;
            __threadfence();
            atomicAdd(&c->barrier_generation, 1u);
        } else {
            long long start = clock64();
            while (*gen == g) {
                if (*(volatile uint32_t*)&c->error) break;
                if (clock64() - start > limit) {
                    atomicExch(&c->error, kErrorBarrierTimeout);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile uint32_t*)&c->error == 0;
}

// Tally: Opaque<NoTally> for scenes without alpha-textured materials;
// kTextures: false for scenes without textured materials (see
// persistent_kernel).  The fused kernel needs ~244 registers unbounded (2
// CTAs per SM); bounded to 8 CTAs of 128 (64 registers) it spills but keeps
// four times the warps resident to hide its traversal latency: 1080p large
// mesh 32.9 -> 40.1 Mpaths/s (3, 4, 5, 6, 10, 12, 16 CTAs: 33.8, 35.5,
// 36.3, 37.3, 39.5, 40.4, 40.5).
template <typename Tally, bool kTextures>
__global__ void __launch_bounds__(128, 8) k_persistent(const __grid_constant__ DeviceScene s,
                                                    const __grid_constant__ RenderParams rp, const TileDev* tile_ptr,
                                                    Counters* c, PathSoA ps, uint32_t* q0, uint32_t* q1,
                                                    uint32_t capacity, float* framebuffer, uint32_t chunk_warps) {
    count_launch(c);
    TileDev tile = *tile_ptr;
    uint32_t n0 = min(tile.width * tile.height, capacity);
    uint32_t sample = c->sample_index;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t lane = threadIdx.x & 31;
    for (uint32_t lp = gid; lp < n0; lp += gridDim.x * blockDim.x) {
        Path path;
        init_path(rp, tile, sample, lp, path);
        store_path(ps, lp, path);
        ps.radiance[lp] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        q0[lp] = lp;
    }
    if (gid == 0) {
        c->persistent_count[0] = n0;
        c->paths += n0;
    }
    if (!grid_barrier(c, gridDim.x)) return;
    unsigned long long shadow_rays = 0;
    for (uint32_t bounce = 0; bounce < rp.max_depth && bounce < kMaxBounces; ++bounce) {
        uint32_t n = *(volatile uint32_t*)&c->persistent_count[bounce];
        if (gid == 0) {
            c->profile[bounce] = n;
            c->extension_rays += n;
        }
        if (n == 0) {
            if (gid == 0)
                for (uint32_t b = bounce + 1; b < rp.max_depth && b < kMaxBounces; ++b) c->profile[b] = 0;
            break;
        }
        uint32_t* cur = (bounce & 1) ? q1 : q0;
        uint32_t* next = (bounce & 1) ? q0 : q1;
        uint32_t* next_count = &c->persistent_count[bounce + 1];
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&c->persistent_work[bounce], 32u * chunk_warps);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= n) break;
            for (uint32_t sub = 0; sub < chunk_warps && base + sub * 32 < n; ++sub) {
                uint32_t i = base + sub * 32 + lane;
                bool alive = false;
                uint32_t p = 0;
                if (i < n) {
                    p = cur[i];
                    Path path = load_path(ps, p);
                    TraceState h;
                    Tally tally;
                    trace_closest(s, path.origin, path.direction, h, tally);
                    SurfaceHit sh;
                    bool did_hit = finish_hit(s, path.origin, path.direction, h.t, h.u, h.v, h.prim, h.inst, sh);
                    InlineSink<Tally> sink;
                    sink.scene = &s;
                    sink.radiance = f4xyz(ps.radiance[p]);
                    sink.killed = false;
                    sink.requests = 0;
                    alive = shade_path<InlineSink<Tally>, kTextures>(s, rp, path, did_hit, sh, sink);
                    alive = alive && !sink.killed;
                    shadow_rays += sink.requests;
                    store_path(ps, p, path);
                    if (alive) {
                        ps.radiance[p] = make_float4(sink.radiance.x, sink.radiance.y, sink.radiance.z, 0.0f);
                    } else {
                        float* f = framebuffer + 3 * size_t(path.pixel);
                        f[0] += sink.radiance.x;
                        f[1] += sink.radiance.y;
                        f[2] += sink.radiance.z;
                    }
                }
                unsigned mask = __ballot_sync(0xffffffffu, alive);
                uint32_t out = 0;
                if (lane == 0 && mask) out = atomicAdd(next_count, uint32_t(__popc(mask)));
                out = __shfl_sync(0xffffffffu, out, 0);
                uint32_t rank = __popc(mask & ((1u << lane) - 1u));
                if (alive && out + rank < capacity) next[out + rank] = p;
            }
        }
        if (!grid_barrier(c, gridDim.x)) return;
    }
    for (int off = 16; off > 0; off >>= 1) shadow_rays += __shfl_down_sync(0xffffffffu, shadow_rays, off);
    if (lane == 0 && shadow_rays) atomicAdd(&c->shadow_rays, shadow_rays);
}

// The persistent kernel for a scene: without the alpha test when no material
// is alpha-textured, without the texture code when none is textured.
const void* persistent_kernel(bool opaque, bool textured) {
    if (!opaque) return reinterpret_cast<const void*>(k_persistent<NoTally, true>);
    return textured ? reinterpret_cast<const void*>(k_persistent<Opaque<NoTally>, true>)
                    : reinterpret_cast<const void*>(k_persistent<Opaque<NoTally>, false>);
}

// The phased persistent kernel (WF_MODE_PERSISTENT renderers): one
// cooperative launch renders one sample of a tile, running the wavefront
// stages -- camera rays, closest hit (per thread at bounce 0, lane refill
// after), material classification and sort, shading with deferred shadow
// rays and caustic gathers, any-hit shadow rays, ordered finalize -- one
// after another over the whole grid, with a bounded grid barrier between
// stages.  The reference's persistent kernel (persistentWavefrontTrace,
// renderer.cu:55-125) instead traces, shades and tests the shadow rays of
// one path in a single fused body; fused, that body needs ~244 registers,
// and bounded for occupancy it spills ~1.6 KB per thread.  Staged, every
// path still sees the same arithmetic in the same order (the stages are
// those of the captured graph), so the sums are unchanged.
struct PhasedBuffers {
    PathSoA ps;
    uint32_t* queue[2];
    float4* hit_a;
    uint32_t* hit_inst;
    float4* terms;
    int4* shade_out;
    float4* shadow_origin;
    float4* shadow_dir;
    uint8_t* shadow_result;
    uint32_t shadow_capacity;
    uint8_t* shade_key;
    uint32_t* shade_order;
    GatherQueue gathers;
    float* framebuffer;
    uint32_t capacity;
    uint32_t refill;
};

// Each stage is an out-of-line call, so the register allocator sees one
// stage at a time instead of every stage's live ranges at once.
#define WF_STAGE static __device__ __noinline__
template <typename Tally, bool kLanes>
WF_STAGE void phased_trace(const DeviceScene& s, const PhasedBuffers& b, uint32_t cur, Counters* c, uint32_t bounce) {
    trace_stage<Tally, kLanes>(s, b.ps, b.queue[cur], &c->queue_count[cur], b.hit_a, b.hit_inst, c, bounce, nullptr,
                               b.refill, nullptr, nullptr);
}
WF_STAGE void phased_classify(const DeviceScene& s, const PhasedBuffers& b, uint32_t cur, Counters* c) {
    classify_stage(s, &c->queue_count[cur], b.hit_a, b.hit_inst, b.shade_key, c);
}
WF_STAGE void phased_scatter(const PhasedBuffers& b, uint32_t cur, Counters* c) {
    scatter_stage(&c->queue_count[cur], b.shade_key, b.shade_order, c);
}
template <bool kTextures>
WF_STAGE void phased_shade(const DeviceScene& s, const RenderParams& rp, const PhasedBuffers& b, uint32_t cur,
                           Counters* c) {
    shade_stage<kTextures>(s, rp, b.ps, b.queue[cur], &c->queue_count[cur], b.hit_a, b.hit_inst, b.terms,
                           b.shade_out, b.shadow_origin, b.shadow_dir, b.shadow_capacity, c,
                           &c->queue_count[cur ^ 1], b.gathers, b.shade_order);
}
WF_STAGE void phased_gather(const RenderParams& rp, const PhasedBuffers& b, Counters* c, bool dense) {
    if (dense)
        gather_dense_stage(rp, b.gathers, b.terms, c);
    else
        gather_stage(rp, b.gathers, b.terms, c);
}
template <typename Tally>
WF_STAGE void phased_shadow(const DeviceScene& s, const PhasedBuffers& b, Counters* c) {
    shadow_stage<Tally>(s, b.shadow_origin, b.shadow_dir, b.shadow_result, c, b.shadow_capacity, nullptr, b.refill);
}
WF_STAGE void phased_finalize(const RenderParams& rp, const PhasedBuffers& b, uint32_t cur, Counters* c,
                              const TileDev* tile_ptr) {
    finalize_stage<false>(b.ps, b.queue[cur], &c->queue_count[cur], b.terms, b.shade_out, b.shadow_result,
                          b.queue[cur ^ 1], &c->queue_count[cur ^ 1], b.capacity, b.framebuffer, &c->work_trace, rp,
                          tile_ptr, c);
}

// CTAs of 128 per SM the phased kernel is bounded to (registers per thread
// = 65536 / (128 x this)); a build setting (make PHASED_CTAS=n).
#ifndef WF_PHASED_CTAS
#define WF_PHASED_CTAS 6
#endif
template <typename Tally, bool kTextures>
__global__ void __launch_bounds__(128, WF_PHASED_CTAS) k_persistent_phased(const __grid_constant__ DeviceScene s,
                                                           const __grid_constant__ RenderParams rp,
                                                           const TileDev* tile_ptr, Counters* c,
                                                           const __grid_constant__ PhasedBuffers b) {
    count_launch(c);
    uint32_t blocks = gridDim.x;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    raygen_stage(rp, tile_ptr, c, b.ps, b.queue[0], b.capacity);
    if (!grid_barrier(c, blocks)) return;
    uint32_t depth = min(rp.max_depth, uint32_t(kMaxBounces));
    for (uint32_t bounce = 0; bounce < depth; ++bounce) {
        uint32_t cur = bounce & 1;
        if (*(volatile uint32_t*)&c->queue_count[cur] == 0) {  // every path ended: the rest are empty
            if (gid == 0)
                for (uint32_t r = bounce; r < depth; ++r) c->profile[r] = 0;
            break;
        }
        if (bounce == 0)
            phased_trace<Tally, false>(s, b, cur, c, bounce);
        else
            phased_trace<Tally, true>(s, b, cur, c, bounce);
        if (!grid_barrier(c, blocks)) return;
        phased_classify(s, b, cur, c);
        if (!grid_barrier(c, blocks)) return;
        phased_scatter(b, cur, c);
        if (!grid_barrier(c, blocks)) return;
        phased_shade<kTextures>(s, rp, b, cur, c);
        if (!grid_barrier(c, blocks)) return;
        if (rp.photons.enabled) {
            phased_gather(rp, b, c, false);
            if (!grid_barrier(c, blocks)) return;
            phased_gather(rp, b, c, true);
        }
        phased_shadow<Tally>(s, b, c);
        if (!grid_barrier(c, blocks)) return;
        phased_finalize(rp, b, cur, c, tile_ptr);
        if (!grid_barrier(c, blocks)) return;
    }
}

const void* phased_kernel(bool opaque, bool textured) {
    if (!opaque) return reinterpret_cast<const void*>(k_persistent_phased<NoTally, true>);
    return textured ? reinterpret_cast<const void*>(k_persistent_phased<Opaque<NoTally>, true>)
                    : reinterpret_cast<const void*>(k_persistent_phased<Opaque<NoTally>, false>);
}

// ---------------------------------------------------------------- batch API
// One closest-hit traversal per thread, bounded to 8 CTAs of 128 per SM (64
// registers; 68 unbounded): 4 M random rays against the 1080p large mesh,
// 365 -> 388 Mrays/s.  k_any_batch already fits 8 CTAs (62 registers).
__global__ void __launch_bounds__(128, 8) k_trace_batch(DeviceScene s, const wf_ray* rays, uint32_t count,
                                                        wf_hit* hits) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    V3 o{rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]};
    V3 d{rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]};
    TraceState h;
    NoTally tally;
    trace_closest(s, o, d, h, tally);
    SurfaceHit sh;
    wf_hit out;
    memset(&out, 0, sizeof(out));
    out.instance = kInvalid;
    out.primitive = kInvalid;
    if (!finish_hit(s, o, d, h.t, h.u, h.v, h.prim, h.inst, sh)) {
        out.t = 1e30f;
        out.material = kInvalid;
        out.light_index = kInvalid;
        out.kind = WF_HIT_NONE;
        hits[i] = out;
        return;
    }
    out.t = sh.t;
    out.position[0] = sh.position.x; out.position[1] = sh.position.y; out.position[2] = sh.position.z;
    out.geometric_normal[0] = sh.geometric_normal.x;
    out.geometric_normal[1] = sh.geometric_normal.y;
    out.geometric_normal[2] = sh.geometric_normal.z;
    out.normal[0] = sh.normal.x; out.normal[1] = sh.normal.y; out.normal[2] = sh.normal.z;
    out.material = sh.material;
    out.light_index = sh.light;
    uint32_t kind = hit_kind(h.prim), index = hit_index(h.prim);
    if (kind == kHitSphere) {
        out.kind = WF_HIT_SPHERE;
        out.primitive = index;
    } else {
        uint32_t original = __float_as_uint(s.triangles[3 * size_t(index)].w) & kTriIndexMask;
        out.primitive = original;
        out.u = h.u;
        out.v = h.v;
        if (kind == kHitMesh) {
            out.kind = WF_HIT_MESH;
            out.instance = h.inst;
        } else {
            out.kind = index >= s.direct_first && index < s.direct_first + s.direct_count ? WF_HIT_TRIANGLE
                                                                                         : WF_HIT_STATIC_TRIANGLE;
        }
    }
    hits[i] = out;
}

__global__ void k_any_batch(DeviceScene s, const wf_ray* rays, const float* max_distance, uint32_t count,
                            uint8_t* occluded) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    V3 o{rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]};
    V3 d{rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]};
    NoTally tally;
    occluded[i] = trace_any(s, o, d, max_distance[i], tally) ? 1 : 0;
}

// ------------------------------------------------------------------ photons
// emitPhotons / tracePhotons, src/renderer/photon_mapping.cu:4-74.  Each
// photon is 4 float4: position (.w = valid), direction (.w = spectral channel),
// flux, rng state (.xy) and specular bounce count (.z).
__global__ void k_emit_photons(const __grid_constant__ DeviceScene s, uint32_t count, uint32_t seed, uint32_t strategy, uint32_t spectral,
                               float4* photons) {
    uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= count || s.light_count == 0) return;
    uint64_t rng = make_rng_state(photon_rng_key(index, seed, strategy), strategy);
    uint32_t candidate = min(uint32_t(random_float(rng, strategy) * s.light_count), s.light_count - 1);
    const Light* cl = &s.lights[candidate];
    uint32_t li = random_float(rng, strategy) < cl->alias_probability ? candidate : cl->alias;
    const Light& light = s.lights[li];
    float root_u = sqrtf(random_float(rng, strategy));
    float v = random_float(rng, strategy);
    V3 point = (1.0f - root_u) * light.v0 + root_u * ((1.0f - v) * light.v1 + v * light.v2);
    Path tmp;
    tmp.rng = rng;
    V3 direction = sample_cosine_hemisphere(light.normal, tmp, strategy);
    rng = tmp.rng;
    const Material& m = s.materials[light.material];
    uint32_t channel = 3;
    V3 flux = m.emission * (light.area * 3.14159265359f / float(count));
    if (spectral) {
        channel = min(uint32_t(random_float(rng, strategy) * 3.0f), 2u);
        flux = V3{0.0f, 0.0f, 0.0f};
        float cf = (channel == 0 ? m.emission.x : channel == 1 ? m.emission.y : m.emission.z) *
                   (light.area * 3.14159265359f * 3.0f / float(count));
        if (channel == 0) flux.x = cf;
        else if (channel == 1) flux.y = cf;
        else flux.z = cf;
    }
    V3 position = point + light.normal * 0.001f;
    float4* ph = photons + 4 * size_t(index);
    ph[0] = make_float4(position.x, position.y, position.z, 0.0f);
    ph[1] = make_float4(direction.x, direction.y, direction.z, __uint_as_float(channel));
    ph[2] = make_float4(flux.x, flux.y, flux.z, 0.0f);
    ph[3] = make_float4(__uint_as_float(uint32_t(rng)), __uint_as_float(uint32_t(rng >> 32)), __uint_as_float(0u), 0.0f);
}

// One photon path per thread, bounded to 8 CTAs of 128 per SM (64
// registers; 96 unbounded): creating the 1080p large-mesh renderer with its
// 2 M-photon map takes 31 ms instead of 34-36 ms.
__global__ void __launch_bounds__(128, 8) k_trace_photons(const __grid_constant__ DeviceScene s, uint32_t count, uint32_t max_depth, uint32_t strategy,
                                float4* photons, uint32_t* stored) {
    uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= count || s.light_count == 0) return;
    float4* ph = photons + 4 * size_t(index);
    float4 p0 = ph[0], p1 = ph[1], p2 = ph[2], p3 = ph[3];
    uint32_t channel = __float_as_uint(p1.w);
    V3 flux = f4xyz(p2);
    Path rngp;
    rngp.rng = uint64_t(__float_as_uint(p3.x)) | (uint64_t(__float_as_uint(p3.y)) << 32);
    uint32_t specular_bounces = 0;
    V3 o = f4xyz(p0), d = f4xyz(p1);
    for (uint32_t depth = 0; depth < max_depth; ++depth) {
        TraceState h;
        NoTally tally;
        trace_closest(s, o, d, h, tally);
        SurfaceHit hit;
        if (!finish_hit(s, o, d, h.t, h.u, h.v, h.prim, h.inst, hit)) return;
        if (hit.material >= s.material_count) return;
        const Material& m = s.materials[hit.material];
        V3 normal = dot(hit.normal, -d) >= 0.0f ? hit.normal : -hit.normal;
        if (m.type == kDiffuse) {
            if (specular_bounces == 0) return;
            V3 back = -d;
            ph[0] = make_float4(hit.position.x, hit.position.y, hit.position.z, 1.0f);
            ph[1] = make_float4(back.x, back.y, back.z, __uint_as_float(channel));
            ph[2] = make_float4(flux.x, flux.y, flux.z, 0.0f);
            ph[3] = make_float4(__uint_as_float(uint32_t(rngp.rng)), __uint_as_float(uint32_t(rngp.rng >> 32)),
                                __uint_as_float(specular_bounces), 0.0f);
            atomicAdd(stored, 1u);
            return;
        }
        V3 direction;
        if (m.type == kMetal) {
            direction = normalize(reflect(normalize(d), normal));
        } else if (m.type == kDielectric) {
            float ior = m.ior;
            if (m.dispersion > 0.0f && channel < 3) ior += (float(channel) - 1.0f) * m.dispersion;
            DielectricInterface b = dielectric_interface(normalize(d), hit.geometric_normal, hit.normal, ior);
            bool reflected = b.reflectance >= 1.0f || b.reflectance > random_float(rngp.rng, strategy);
            direction = reflected ? b.reflection : b.transmission;
        } else {
            direction = sample_cosine_hemisphere(normal, rngp, strategy);
        }
        if (m.type == kMetal || m.type == kDielectric) ++specular_bounces;
        flux = hadamard(flux, m.albedo);
        o = offset_ray_origin(hit.position, hit.geometric_normal, direction, hit.t);
        d = direction;
    }
}

// An order-preserving map of floats onto uint32, so the photon bounds can be
// taken with integer atomicMin / atomicMax; build_photon_map decodes it.
WF_DEV uint32_t float_order(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_photon_bounds(const float4* photons, uint32_t count, uint32_t* bounds) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float4 p = photons[4 * size_t(i)];
    if (p.w != 1.0f) return;
    atomicMin(&bounds[0], float_order(p.x));
    atomicMin(&bounds[1], float_order(p.y));
    atomicMin(&bounds[2], float_order(p.z));
    atomicMax(&bounds[3], float_order(p.x));
    atomicMax(&bounds[4], float_order(p.y));
    atomicMax(&bounds[5], float_order(p.z));
}

// buildPhotonGrid cell rule (photon_mapping.cu:76-89); key = cell, then
// descending photon index (the order serial insertion leaves in each list).
__global__ void k_photon_keys(const float4* photons, uint32_t count, uint32_t padded, PhotonGridView g,
                              unsigned long long* keys) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= padded) return;
    unsigned long long key = ~0ull;
    if (i < count) {
        float4 p = photons[4 * size_t(i)];
        if (p.w == 1.0f) {
            V3 extent = g.maximum - g.minimum;
            V3 offset = V3{p.x, p.y, p.z} - g.minimum;
            V3 nrm{offset.x / extent.x, offset.y / extent.y, offset.z / extent.z};
            int res = int(g.resolution);
            int x = min(max(int(nrm.x * g.resolution), 0), res - 1);
            int y = min(max(int(nrm.y * g.resolution), 0), res - 1);
            int z = min(max(int(nrm.z * g.resolution), 0), res - 1);
            bool inside = !(nrm.x < 0.0f || nrm.y < 0.0f || nrm.z < 0.0f || nrm.x > 1.0f || nrm.y > 1.0f || nrm.z > 1.0f);
            if (inside) {
                uint32_t cell = (uint32_t(z) * g.resolution + uint32_t(y)) * g.resolution + uint32_t(x);
                key = (uint64_t(cell) << 32) | uint64_t(0xffffffffu - i);
            }
        }
    }
    keys[i] = key;
}

__global__ void k_bitonic(unsigned long long* keys, uint32_t j, uint32_t k, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t l = i ^ j;
    if (l > i) {
        unsigned long long a = keys[i], b = keys[l];
        bool ascending = (i & k) == 0;
        if ((a > b) == ascending) {
            keys[i] = b;
            keys[l] = a;
        }
    }
}

__global__ void k_photon_scatter(const unsigned long long* keys, uint32_t padded, const float4* photons,
                                 float4* pos, float4* dir, float4* flux, uint32_t* cell_start, uint32_t* cell_end) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= padded) return;
    unsigned long long key = keys[j];
    if (key == ~0ull) return;
    uint32_t index = 0xffffffffu - uint32_t(key);
    uint32_t cell = uint32_t(key >> 32);
    const float4* ph = photons + 4 * size_t(index);
    pos[j] = ph[0];
    dir[j] = ph[1];
    flux[j] = ph[2];
    if (j == 0 || uint32_t(keys[j - 1] >> 32) != cell) cell_start[cell] = j;
    if (j + 1 == padded || keys[j + 1] == ~0ull || uint32_t(keys[j + 1] >> 32) != cell) cell_end[cell] = j + 1;
}

__global__ void k_cell_counts(const uint32_t* start, uint32_t* end_to_count, uint32_t cells) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < cells) end_to_count[c] = end_to_count[c] - start[c];
}

template <typename T>
cudaError_t alloc(wf_renderer* r, T** p, size_t count) {
    size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
    cudaError_t e = device_alloc(reinterpret_cast<void**>(p), bytes);
    if (e == cudaSuccess) {
        r->allocations.push_back(*p);
        r->device_bytes += bytes;
    }
    return e;
}

uint32_t grid_for(const wf_renderer* r, uint32_t work, uint32_t block) {
    uint32_t g = (work + block - 1) / block;
    return std::max(1u, std::min(g, r->grid_cap));
}

// Bounce kernels fetch work dynamically (per-warp chunks or a grid-stride
// loop), so one full wave of resident CTAs covers any queue; a larger grid
// only adds CTAs that find nothing to do.
uint32_t grid(const wf_renderer* r, int kernel, uint32_t work, uint32_t block) {
    uint32_t g = grid_for(r, work, block);
    return r->grid_resident[kernel] ? std::min(g, r->grid_resident[kernel]) : g;
}

template <typename K>
cudaError_t resident_grid(wf_renderer* r, int kernel, K* fn, uint32_t block) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, int(block), 0);
    if (e == cudaSuccess) r->grid_resident[kernel] = uint32_t(std::max(per_sm, 1)) * uint32_t(r->sm_count);
    return e;
}

wf_status build_photon_map(wf_renderer* r) {
    const wf_render_config& c = r->config;
    const DeviceScene& s = r->scene->view;
    uint32_t n = c.photon_count;
    r->photons_emitted = n;
    if (s.light_count == 0 || n == 0) {
        r->params.photons.enabled = 0;
        return WF_OK;
    }
    WF_CUDA(alloc(r, &r->photon_raw, size_t(n) * 4));
    uint32_t* stored = nullptr;
    WF_CUDA(alloc(r, &stored, 8));
    WF_CUDA(cudaMemsetAsync(r->photon_raw, 0, sizeof(float4) * 4 * size_t(n), r->stream));
    WF_CUDA(cudaMemsetAsync(stored, 0, 8 * sizeof(uint32_t), r->stream));
    uint32_t block = 128;
    k_emit_photons<<<(n + block - 1) / block, block, 0, r->stream>>>(s, n, c.photon_seed, c.rng, c.spectral, r->photon_raw);
    k_trace_photons<<<(n + block - 1) / block, block, 0, r->stream>>>(s, n, c.photon_max_depth, c.rng, r->photon_raw,
                                                                     stored);
    WF_CUDA(cudaGetLastError());
    PhotonGridView& g = r->params.photons;
    g.resolution = c.photon_grid_resolution ? c.photon_grid_resolution : 64;
    bool derive = c.photon_grid_min[0] == c.photon_grid_max[0] && c.photon_grid_min[1] == c.photon_grid_max[1] &&
                  c.photon_grid_min[2] == c.photon_grid_max[2];
    if (derive) {
        uint32_t init[8] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u, 0u};
        uint32_t* bounds = stored + 2;
        WF_CUDA(cudaMemcpyAsync(bounds, init, 6 * sizeof(uint32_t), cudaMemcpyHostToDevice, r->stream));
        k_photon_bounds<<<(n + block - 1) / block, block, 0, r->stream>>>(r->photon_raw, n, bounds);
    }
    uint32_t host[8];
    WF_CUDA(cudaMemcpyAsync(host, stored, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, r->stream));
    WF_CUDA(cudaStreamSynchronize(r->stream));
    r->photons_stored = host[0];
    if (derive) {
        auto dec = [](uint32_t u) {
            uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
            float f;
            std::memcpy(&f, &b, 4);
            return f;
        };
        if (host[0] == 0) {
            g.minimum = V3{-1, -1, -1};
            g.maximum = V3{1, 1, 1};
        } else {
            g.minimum = V3{dec(host[2]), dec(host[3]), dec(host[4])};
            g.maximum = V3{dec(host[5]), dec(host[6]), dec(host[7])};
            // Degenerate axes get unit extent so the normalization stays finite.
            if (!(g.maximum.x > g.minimum.x)) g.maximum.x = g.minimum.x + 1.0f;
            if (!(g.maximum.y > g.minimum.y)) g.maximum.y = g.minimum.y + 1.0f;
            if (!(g.maximum.z > g.minimum.z)) g.maximum.z = g.minimum.z + 1.0f;
        }
    } else {
        g.minimum = V3{c.photon_grid_min[0], c.photon_grid_min[1], c.photon_grid_min[2]};
        g.maximum = V3{c.photon_grid_max[0], c.photon_grid_max[1], c.photon_grid_max[2]};
    }
    uint32_t padded = 1;
    while (padded < n) padded <<= 1;
    unsigned long long* keys = nullptr;
    uint32_t cells = g.resolution * g.resolution * g.resolution;
    float4 *pos = nullptr, *dir = nullptr, *flux = nullptr;
    uint32_t *start = nullptr, *end = nullptr;
    WF_CUDA(alloc(r, &keys, padded));
    WF_CUDA(alloc(r, &pos, padded));
    WF_CUDA(alloc(r, &dir, padded));
    WF_CUDA(alloc(r, &flux, padded));
    WF_CUDA(alloc(r, &start, cells));
    WF_CUDA(alloc(r, &end, cells));
    WF_CUDA(cudaMemsetAsync(start, 0, sizeof(uint32_t) * cells, r->stream));
    WF_CUDA(cudaMemsetAsync(end, 0, sizeof(uint32_t) * cells, r->stream));
    uint32_t sb = 256;
    k_photon_keys<<<(padded + sb - 1) / sb, sb, 0, r->stream>>>(r->photon_raw, n, padded, g, keys);
    for (uint32_t k = 2; k <= padded; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1)
            k_bitonic<<<(padded + sb - 1) / sb, sb, 0, r->stream>>>(keys, j, k, padded);
    k_photon_scatter<<<(padded + sb - 1) / sb, sb, 0, r->stream>>>(keys, padded, r->photon_raw, pos, dir, flux, start,
                                                                   end);
    k_cell_counts<<<(cells + sb - 1) / sb, sb, 0, r->stream>>>(start, end, cells);
    WF_CUDA(cudaGetLastError());
    g.position = pos;
    g.direction = dir;
    g.flux = flux;
    g.cell_start = start;
    g.cell_count = end;
    g.enabled = c.caustic_gather ? 1u : 0u;
    return WF_OK;
}

// k_trace / k_shadow for this renderer's scene: the Opaque<> variants (the
// per-hit alpha-texture test compiled out, fewer registers) unless some
// material of the scene is alpha-textured.
template <typename Tally, bool kLanes, typename... A>
void launch_trace(const wf_renderer* r, uint32_t grid_size, uint32_t block, cudaStream_t st, A... args) {
    if constexpr (!kLanes) {
        if (r->opaque)
            k_trace_camera<Opaque<Tally>><<<grid_size, block, 0, st>>>(args...);
        else
            k_trace_camera<Tally><<<grid_size, block, 0, st>>>(args...);
    } else if (r->opaque) {
        k_trace<Opaque<Tally>, kLanes><<<grid_size, block, 0, st>>>(args...);
    } else {
        k_trace<Tally, kLanes><<<grid_size, block, 0, st>>>(args...);
    }
}
// k_shade with the texture code only for scenes that have textured materials.
template <typename... A>
void launch_shade(const wf_renderer* r, uint32_t grid_size, uint32_t block, cudaStream_t st, A... args) {
    if (r->textured)
        k_shade<true><<<grid_size, block, 0, st>>>(args...);
    else
        k_shade<false><<<grid_size, block, 0, st>>>(args...);
}
template <typename Tally, typename... A>
void launch_shadow(const wf_renderer* r, uint32_t grid_size, uint32_t block, cudaStream_t st, A... args) {
    if (r->opaque)
        k_shadow<Opaque<Tally>><<<grid_size, block, 0, st>>>(args...);
    else
        k_shadow<Tally><<<grid_size, block, 0, st>>>(args...);
}

wf_status capture_graph(wf_renderer* r) {
    const DeviceScene& s = r->scene->view;
    cudaStream_t st = r->stream;
    WF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    uint32_t cap = r->capacity;
    k_raygen<<<grid_for(r, cap, 256), 256, 0, st>>>(r->params, r->tile, r->counters, r->paths, r->queue[0], cap);
    for (uint32_t b = 0; b < r->config.max_depth; ++b) {
        uint32_t cur = b & 1, nxt = cur ^ 1;
        uint32_t* cur_count = &r->counters->queue_count[cur];
        uint32_t* next_count = &r->counters->queue_count[nxt];
        if (b == 0)
            launch_trace<NoTally, false>(r, grid(r, 5, cap, r->block_camera), r->block_camera, st, 
                s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, b, nullptr, r->refill,
                nullptr, nullptr);
        else
            launch_trace<NoTally, true>(r, grid(r, 0, cap, r->block_trace), r->block_trace, st, 
                s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, b, nullptr, r->refill,
                nullptr, nullptr);
        if (r->sort_shading) {
            k_classify<<<grid(r, 3, cap, 256), 256, 0, st>>>(s, cur_count, r->hit_a, r->hit_inst, r->shade_key,
                                                              r->counters);
            k_scatter<<<grid(r, 3, cap, 256), 256, 0, st>>>(cur_count, r->shade_key, r->shade_order, r->counters);
        }
        launch_shade(r, grid(r, 1, cap, r->block_shade), r->block_shade, st, 
            s, r->params, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->terms, r->shade_out,
            r->shadow_origin, r->shadow_dir, r->shadow_capacity, r->counters, next_count, r->gathers,
            r->sort_shading ? r->shade_order : nullptr);
        bool fork = r->params.photons.enabled != 0;
        if (fork) {  // gathers on a parallel branch: they and the shadow rays write different buffers
            WF_CUDA(cudaEventRecord(r->fork_event, st));
            WF_CUDA(cudaStreamWaitEvent(r->side, r->fork_event, 0));
            k_gather<<<grid(r, 4, cap, r->block_gather), r->block_gather, 0, r->side>>>(r->params, r->gathers,
                                                                                        r->terms, r->counters);
            k_gather_dense<<<grid(r, 4, cap, r->block_gather), r->block_gather, 0, r->side>>>(
                r->params, r->gathers, r->terms, r->counters);
            WF_CUDA(cudaEventRecord(r->join_event, r->side));
        }
        launch_shadow<NoTally>(r, grid(r, 2, r->shadow_capacity, r->block_trace), r->block_trace, st, 
            s, r->shadow_origin, r->shadow_dir, r->shadow_result, r->counters, r->shadow_capacity, nullptr, r->refill);
        if (fork) WF_CUDA(cudaStreamWaitEvent(st, r->join_event, 0));
        k_finalize<false><<<grid(r, 3, cap, r->block_finalize), r->block_finalize, 0, st>>>(
            r->paths, r->queue[cur], cur_count, r->terms, r->shade_out, r->shadow_result, r->queue[nxt], next_count,
            cap, r->framebuffer, &r->counters->work_trace, r->params, r->tile, r->counters);
    }
    if (r->wave > 1)
        k_accumulate_wave<<<grid_for(r, r->tile_capacity, 256), 256, 0, st>>>(r->paths, r->tile, r->framebuffer,
                                                                                r->counters);
    k_advance<<<1, 1, 0, st>>>(r->counters, r->tile);
    cudaError_t e = cudaStreamEndCapture(st, &r->graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    WF_CUDA(cudaGraphInstantiate(&r->graph_exec, r->graph, 0));
    return WF_OK;
}

// Streaming graph: raygen, then a device-side WHILE node whose body runs two
// bounces (queue 0 -> 1 -> 0) and re-arms itself while queue 0 is non-empty,
// then the sample-index advance.  Built with cudaStreamBeginCaptureToGraph
// into the parent graph and the conditional node's body graph.
wf_status capture_stream_graph(wf_renderer* r) {
    const DeviceScene& s = r->scene->view;
    cudaStream_t st = r->stream;
    uint32_t cap = r->capacity;
    WF_CUDA(cudaGraphCreate(&r->graph, 0));
    WF_CUDA(cudaStreamBeginCaptureToGraph(st, r->graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    k_raygen_stream<<<grid_for(r, cap, 256), 256, 0, st>>>(r->params, r->tile, r->counters, r->paths, r->queue[0],
                                                            cap);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &captured);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (stream prologue)");
    size_t nodes = 0;
    WF_CUDA(cudaGraphGetNodes(r->graph, nullptr, &nodes));
    if (nodes != 1) return fail(WF_ERR_CUDA, "unexpected streaming prologue graph (%zu nodes)", nodes);
    cudaGraphNode_t raygen_node = nullptr;
    WF_CUDA(cudaGraphGetNodes(r->graph, &raygen_node, &nodes));

    cudaGraphConditionalHandle handle;
    WF_CUDA(cudaGraphConditionalHandleCreate(&handle, r->graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop_node = nullptr;
    WF_CUDA(cudaGraphAddNode(&loop_node, r->graph, &raygen_node, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];

    WF_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    for (uint32_t cur = 0; cur < 2; ++cur) {
        uint32_t nxt = cur ^ 1;
        uint32_t* cur_count = &r->counters->queue_count[cur];
        uint32_t* next_count = &r->counters->queue_count[nxt];
        // The survivors and the camera rays of slots that started a sample
        // (see trace_stage): lane refill over both, or per thread over the
        // camera rays when nothing survived.  The launch with nothing to do
        // exits at once.
        uint32_t* camera = &r->counters->camera_count[cur];
        launch_trace<NoTally, false>(r, grid(r, 5, cap, r->block_camera), r->block_camera, st,
            s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, kMaxBounces, nullptr,
            r->refill, camera, &r->counters->work_camera);
        launch_trace<NoTally, true>(r, grid(r, 0, cap, r->block_trace), r->block_trace, st,
            s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, kMaxBounces, nullptr, r->refill,
            camera, nullptr);
        k_merge_camera<<<1, 1, 0, st>>>(r->counters, cur);
        if (r->sort_shading) {
            k_classify<<<grid(r, 3, cap, 256), 256, 0, st>>>(s, cur_count, r->hit_a, r->hit_inst, r->shade_key,
                                                              r->counters);
            k_scatter<<<grid(r, 3, cap, 256), 256, 0, st>>>(cur_count, r->shade_key, r->shade_order, r->counters);
        }
        launch_shade(r, grid(r, 1, cap, r->block_shade), r->block_shade, st, 
            s, r->params, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->terms, r->shade_out,
            r->shadow_origin, r->shadow_dir, r->shadow_capacity, r->counters, next_count, r->gathers,
            r->sort_shading ? r->shade_order : nullptr);
        bool fork = r->params.photons.enabled != 0;
        if (fork) {  // gathers on a parallel branch: they and the shadow rays write different buffers
            WF_CUDA(cudaEventRecord(r->fork_event, st));
            WF_CUDA(cudaStreamWaitEvent(r->side, r->fork_event, 0));
            k_gather<<<grid(r, 4, cap, r->block_gather), r->block_gather, 0, r->side>>>(r->params, r->gathers,
                                                                                        r->terms, r->counters);
            k_gather_dense<<<grid(r, 4, cap, r->block_gather), r->block_gather, 0, r->side>>>(
                r->params, r->gathers, r->terms, r->counters);
            WF_CUDA(cudaEventRecord(r->join_event, r->side));
        }
        launch_shadow<NoTally>(r, grid(r, 2, r->shadow_capacity, r->block_trace), r->block_trace, st, 
            s, r->shadow_origin, r->shadow_dir, r->shadow_result, r->counters, r->shadow_capacity, nullptr, r->refill);
        if (fork) WF_CUDA(cudaStreamWaitEvent(st, r->join_event, 0));
        k_finalize<true><<<grid(r, 3, cap, r->block_finalize), r->block_finalize, 0, st>>>(
            r->paths, r->queue[cur], cur_count, r->terms, r->shade_out, r->shadow_result, r->queue[nxt], next_count,
            cap, r->framebuffer, &r->counters->work_trace, r->params, r->tile, r->counters);
        k_regenerate<<<grid(r, 3, cap, 256), 256, 0, st>>>(r->params, r->tile, r->counters, r->paths, r->queue[nxt],
                                                           next_count, &r->counters->camera_count[nxt], cap,
                                                           r->regenerate_percent);
    }
    k_stream_condition<<<1, 1, 0, st>>>(handle, r->counters, r->tile, r->config.max_depth);
    e = cudaStreamEndCapture(st, &captured);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (stream body)");

    WF_CUDA(cudaStreamBeginCaptureToGraph(st, r->graph, &loop_node, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    k_advance<<<1, 1, 0, st>>>(r->counters, r->tile);
    e = cudaStreamEndCapture(st, &captured);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (stream epilogue)");
    WF_CUDA(cudaGraphInstantiate(&r->graph_exec, r->graph, 0));
    return WF_OK;
}

// Grid of one persistent launch over `paths` paths: the configured grid, or
// by default the resident grid trimmed for small tiles to one CTA per 128
// paths, but never below 4 CTAs per SM.  Every CTA joins each bounce's grid
// barrier, so on a small tile a full resident grid costs more in barriers
// than its idle warps give (256x256 Cornell box: 592 CTAs 128.7 Mpaths/s,
// 1184 CTAs 105.4); large tiles keep the whole resident grid.
uint32_t persistent_grid(uint32_t configured, uint32_t resident, uint32_t sm_count, uint64_t paths) {
    if (configured) return std::max(1u, std::min(configured, resident));
    uint64_t wanted = std::max<uint64_t>(4ull * sm_count, (paths + 127) / 128);
    return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(wanted, resident)));
}

// One cooperative launch of the phased persistent kernel over `paths`
// paths of the current tile (the tile record is already on the device).
cudaError_t launch_phased(wf_renderer* r, cudaStream_t st, uint64_t paths) {
    cudaError_t e = cudaMemsetAsync(&r->counters->barrier_count, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    DeviceScene s = r->scene->view;
    RenderParams rp = r->params;
    const TileDev* tp = r->tile;
    Counters* c = r->counters;
    PhasedBuffers b{};
    b.ps = r->paths;
    b.queue[0] = r->queue[0];
    b.queue[1] = r->queue[1];
    b.hit_a = r->hit_a;
    b.hit_inst = r->hit_inst;
    b.terms = r->terms;
    b.shade_out = r->shade_out;
    b.shadow_origin = r->shadow_origin;
    b.shadow_dir = r->shadow_dir;
    b.shadow_result = r->shadow_result;
    b.shadow_capacity = r->shadow_capacity;
    b.shade_key = r->shade_key;
    b.shade_order = r->shade_order;
    b.gathers = r->gathers;
    b.framebuffer = r->framebuffer;
    b.capacity = r->capacity;
    b.refill = r->refill;
    void* args[] = {&s, &rp, &tp, &c, &b};
    uint32_t blocks = persistent_grid(r->config.persistent_blocks, r->phased_blocks, r->sm_count,
                                      std::min<uint64_t>(paths, r->capacity));
    return cudaLaunchCooperativeKernel(phased_kernel(r->opaque, r->textured), dim3(blocks),
                                       dim3(r->persistent_block_size), args, 0, st);
}

// One cooperative launch of the fused persistent kernel (k_persistent).
cudaError_t launch_fused(wf_renderer* r, cudaStream_t st, uint64_t paths) {
    cudaError_t e = cudaMemsetAsync(r->counters->persistent_count, 0, sizeof(uint32_t) * 2 * (kMaxBounces + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(&r->counters->barrier_count, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    DeviceScene s = r->scene->view;
    RenderParams rp = r->params;
    const TileDev* tp = r->tile;
    Counters* c = r->counters;
    PathSoA ps = r->paths;
    uint32_t* q0 = r->queue[0];
    uint32_t* q1 = r->queue[1];
    uint32_t cap = r->capacity;
    float* fb = r->framebuffer;
    uint32_t chunk = r->chunk;
    void* args[] = {&s, &rp, &tp, &c, &ps, &q0, &q1, &cap, &fb, &chunk};
    uint32_t blocks = persistent_grid(r->config.persistent_blocks, r->persistent_blocks, r->sm_count,
                                      std::min<uint64_t>(paths, r->capacity));
    return cudaLaunchCooperativeKernel(persistent_kernel(r->opaque, r->textured), dim3(blocks),
                                       dim3(r->persistent_block_size), args, 0, st);
}

// The persistent schedule's launch for a tile of `paths` paths: the staged
// kernel pays a grid barrier per stage, which a small tile does not amortise
// (256x256 Cornell box: fused 127, staged 72 Mpaths/s), while on large tiles
// the fused body's spills dominate (1080p large mesh: fused 47, staged 84).
constexpr uint64_t kStagedMinPaths = 262144;
cudaError_t launch_persistent(wf_renderer* r, cudaStream_t st, uint64_t paths) {
    uint32_t k = r->config.persistent_stages;
    bool staged = k == WF_PERSISTENT_STAGED || r->wave > 1 || (k == WF_PERSISTENT_AUTO && paths >= kStagedMinPaths);
    return staged ? launch_phased(r, st, paths) : launch_fused(r, st, paths);
}

wf_status launch_tile(wf_renderer* r, const TileDev& tile) {
    WF_CUDA(cudaMemcpyAsync(r->tile, &tile, sizeof(TileDev), cudaMemcpyHostToDevice, r->stream));
    r->last_tile_width = tile.width;
    r->last_tile_height = tile.height;
    if (r->config.mode != WF_MODE_PERSISTENT) {
        WF_CUDA(cudaGraphLaunch(r->graph_exec, r->stream));
        return WF_OK;
    }
    WF_CUDA(launch_persistent(r, r->stream, uint64_t(tile.width) * tile.height * tile.samples));
    if (tile.samples > 1)
        k_accumulate_wave<<<grid_for(r, r->tile_capacity, 256), 256, 0, r->stream>>>(r->paths, r->tile,
                                                                                     r->framebuffer, r->counters);
    k_advance<<<1, 1, 0, r->stream>>>(r->counters, r->tile);
    WF_CUDA(cudaGetLastError());
    return WF_OK;
}

}  // namespace

// The config checks of RenderDriver::validateConfiguration and prepare
// (render_driver.cu:104-147,429-437) that every render entry point makes,
// plus this renderer's own fields.
wf_status check_render_config(const wf_scene* scene, const wf_render_config& c) {
    if (!std::isfinite(c.indirect_clamp) || c.indirect_clamp < 0.0f)
        return fail(WF_ERR_INVALID_ARG, "Indirect radiance clamp must be finite and nonnegative");
    if (c.width == 0 || c.height == 0) return fail(WF_ERR_INVALID_ARG, "Render dimensions must be greater than zero");
    if (uint64_t(c.width) * c.height > 0xffffffffull)
        return fail(WF_ERR_INVALID_ARG, "Render dimensions exceed the supported queue index range");
    if (c.max_depth == 0) return fail(WF_ERR_INVALID_ARG, "maximum depth must be greater than zero");
    if (c.max_depth > kMaxBounces) return fail(WF_ERR_INVALID_ARG, "maximum depth above %d", kMaxBounces);
    if (c.block_size > 1024 || c.block_size % 32)
        return fail(WF_ERR_INVALID_ARG, "CUDA block size must be a multiple of 32 up to 1024 (0 = default)");
    if (c.mode > WF_MODE_STREAM || c.rng > WF_RNG_PCG32 || c.debug > WF_DEBUG_SHADING_NORMAL)
        return fail(WF_ERR_INVALID_ARG, "unknown mode, rng strategy or debug view");
    if (c.caustics && c.photon_count == 0)
        return fail(WF_ERR_INVALID_ARG, "Photon count must be greater than zero when caustics are enabled");
    if (!(c.gather_radius > 0.0f))
        return fail(WF_ERR_INVALID_ARG, "Caustic gather radius must be greater than zero");
    if (c.refill_threshold > 32) return fail(WF_ERR_INVALID_ARG, "refill threshold must be between 0 and 32");
    if (c.samples_per_wave > 1024) return fail(WF_ERR_INVALID_ARG, "samples_per_wave must be at most 1024");
    if (scene->view.punctual_count - scene->view.directional_count > 0 && scene->view.directional_count > 2)
        return fail(WF_ERR_UNSUPPORTED, "more than two directional lights");
    return WF_OK;
}

namespace {
// external_framebuffer: render into this buffer instead of allocating one;
// photon_source: reuse that renderer's photon map instead of building one.
wf_status renderer_create_impl(const wf_scene* scene, const wf_camera* camera, const wf_render_config* cfg,
                               void* stream, wf_renderer** out, float* external_framebuffer,
                               const wf_renderer* photon_source) {
    if (!scene || !camera || !cfg || !out) return fail(WF_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    const wf_render_config& c = *cfg;
    if (wf_status e = check_render_config(scene, c)) return e;
    uint64_t pixels = uint64_t(c.width) * c.height;
    uint64_t capacity = (c.tile_width && c.tile_height) ? uint64_t(c.tile_width) * c.tile_height : pixels;
    if (capacity > 0xffffffffull)
        return fail(WF_ERR_INVALID_ARG, "Render dimensions exceed the supported queue index range");

    // A creation that fails part way frees what it had made: renderer_destroy
    // takes a partly built renderer.
    std::unique_ptr<wf_renderer, wf_status (*)(wf_renderer*)> r(new wf_renderer(), renderer_destroy);
    r->scene = scene;
    r->config = c;
    r->tile_capacity = uint32_t(std::min(capacity, pixels));
    // waves: graph mode, and the staged persistent kernel (the fused one
    // adds each path to the framebuffer itself)
    bool waves = c.mode == WF_MODE_GRAPH || (c.mode == WF_MODE_PERSISTENT && c.persistent_stages != WF_PERSISTENT_FUSED);
    r->wave = waves && c.samples_per_wave > 1 ? c.samples_per_wave : 1u;
    if (uint64_t(r->tile_capacity) * r->wave > 0xffffffffull)
        return fail(WF_ERR_INVALID_ARG, "samples_per_wave x tile pixels exceeds the supported queue index range");
    r->capacity = r->tile_capacity * r->wave;
    WF_CUDA(cudaGetDevice(&r->device));
    WF_CUDA(cudaDeviceGetAttribute(&r->sm_count, cudaDevAttrMultiProcessorCount, r->device));
    r->grid_cap = uint32_t(r->sm_count) * 64;
    // The CTA size setting applies to the lane-refill trace and shadow
    // kernels; shading and camera rays keep the 128 their register bounds
    // are written for.
    if (c.block_size) r->block_trace = c.block_size;
    r->refill = c.refill_threshold ? c.refill_threshold : 8u;
    r->regenerate_percent = c.regenerate_percent ? std::min(c.regenerate_percent, 100u) : kDefaultRegeneratePercent;
    r->opaque = !scene->alpha_textures;
    r->textured = scene->textured;
    // Sorting by category pays only when hits can need different long
    // shading branches: with one of diffuse / metal / dielectric / other
    // (misses and emitters are short) the sort's two launches per bounce
    // would buy nothing.
    r->sort_shading = __builtin_popcount(scene->material_categories & 0x3cu) > 1;
    if (stream) {
        r->stream = static_cast<cudaStream_t>(stream);
    } else {
        WF_CUDA(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
        r->own_stream = true;
    }
    RenderParams& rp = r->params;
    rp.width = c.width;
    rp.height = c.height;
    rp.max_depth = c.max_depth;
    rp.rr_start = c.rr_start_depth;
    rp.rng = c.rng;
    rp.debug = c.debug;
    rp.clamp = c.indirect_clamp;
    rp.gather_radius = c.gather_radius;
    rp.camera.position = V3{camera->position[0], camera->position[1], camera->position[2]};
    rp.camera.forward = V3{camera->forward[0], camera->forward[1], camera->forward[2]};
    rp.camera.right = V3{camera->right[0], camera->right[1], camera->right[2]};
    rp.camera.up = V3{camera->up[0], camera->up[1], camera->up[2]};
    rp.camera.aspect_ratio = camera->aspect_ratio;
    rp.camera.tan_half_fov = wfm::tanf(camera->vertical_fov * 0.5f);
    rp.photons = PhotonGridView{};

    uint32_t cap = r->capacity;
    wf_renderer* rr = r.get();
    WF_CUDA(alloc(rr, &r->paths.origin, cap));
    WF_CUDA(alloc(rr, &r->paths.direction, cap));
    WF_CUDA(alloc(rr, &r->paths.throughput, cap));
    WF_CUDA(alloc(rr, &r->paths.radiance, cap));
    WF_CUDA(alloc(rr, &r->paths.info, cap));
    WF_CUDA(alloc(rr, &r->paths.rng, cap));
    WF_CUDA(alloc(rr, &r->queue[0], cap));
    WF_CUDA(alloc(rr, &r->queue[1], cap));
    WF_CUDA(alloc(rr, &r->counters, 1));
    WF_CUDA(alloc(rr, &r->tile, 1));
    WF_CUDA(cudaMemsetAsync(r->counters, 0, sizeof(Counters), r->stream));
    if (external_framebuffer) {
        r->framebuffer = external_framebuffer;
        r->external_framebuffer = true;
    } else {
        WF_CUDA(alloc(rr, &r->framebuffer, size_t(pixels) * 3));
        WF_CUDA(cudaMemsetAsync(r->framebuffer, 0, sizeof(float) * 3 * size_t(pixels), r->stream));
    }
    {  // stage buffers: every schedule runs the wavefront stages
        uint32_t requests_per_path = 5u + scene->view.directional_count;
        uint64_t shadow = uint64_t(cap) * requests_per_path;
        if (c.shadow_queue_capacity && c.shadow_queue_capacity < shadow) shadow = c.shadow_queue_capacity;
        if (shadow > 0xffffffffull) shadow = 0xffffffffull;
        r->shadow_capacity = uint32_t(shadow);
        WF_CUDA(alloc(rr, &r->hit_a, cap));
        WF_CUDA(alloc(rr, &r->hit_inst, cap));
        WF_CUDA(alloc(rr, &r->terms, size_t(cap) * kMaxTerms));
        WF_CUDA(alloc(rr, &r->shade_out, cap));
        WF_CUDA(alloc(rr, &r->shade_key, cap));
        WF_CUDA(alloc(rr, &r->shade_order, cap));
        WF_CUDA(alloc(rr, &r->shadow_origin, r->shadow_capacity));
        WF_CUDA(alloc(rr, &r->shadow_dir, r->shadow_capacity));
        WF_CUDA(alloc(rr, &r->shadow_result, r->shadow_capacity));
        if (c.mode == WF_MODE_STREAM) {
            WF_CUDA(alloc(rr, &r->paths.slot_sample, cap));
            WF_CUDA(alloc(rr, &r->paths.wait, cap));
        }
        if (c.caustics) {
            WF_CUDA(alloc(rr, &r->gathers.position, cap));
            WF_CUDA(alloc(rr, &r->gathers.normal, cap));
            WF_CUDA(alloc(rr, &r->gathers.throughput, cap));
            WF_CUDA(alloc(rr, &r->gathers.albedo, cap));
            r->gathers.count = &r->counters->gather_count;
            r->gathers.capacity = cap;
            WF_CUDA(alloc(rr, &r->gathers.dense, cap));
            r->gathers.dense_count = &r->counters->dense_count;
            WF_CUDA(resident_grid(rr, 4, k_gather, r->block_gather));
        }
    }
    if (c.mode != WF_MODE_PERSISTENT) {
        WF_CUDA(r->opaque ? resident_grid(rr, 0, k_trace<Opaque<NoTally>>, r->block_trace)
                          : resident_grid(rr, 0, k_trace<NoTally>, r->block_trace));
        WF_CUDA(r->opaque ? resident_grid(rr, 5, k_trace_camera<Opaque<NoTally>>, r->block_camera)
                          : resident_grid(rr, 5, k_trace_camera<NoTally>, r->block_camera));
        WF_CUDA(r->textured ? resident_grid(rr, 1, k_shade<true>, r->block_shade)
                            : resident_grid(rr, 1, k_shade<false>, r->block_shade));
        WF_CUDA(r->opaque ? resident_grid(rr, 2, k_shadow<Opaque<NoTally>>, r->block_trace)
                          : resident_grid(rr, 2, k_shadow<NoTally>, r->block_trace));
        WF_CUDA(resident_grid(rr, 3, k_finalize<true>, r->block_finalize));
    } else {
        int cooperative = 0;
        WF_CUDA(cudaDeviceGetAttribute(&cooperative, cudaDevAttrCooperativeLaunch, r->device));
        if (!cooperative) return fail(WF_ERR_UNSUPPORTED, "device does not support cooperative launches");
        if (c.persistent_stages > WF_PERSISTENT_STAGED)
            return fail(WF_ERR_INVALID_ARG, "unknown persistent kernel %u", c.persistent_stages);
        r->persistent_block_size = 128;
        int per_sm = 0;
        WF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_kernel(r->opaque, r->textured),
                                                              int(r->persistent_block_size), 0));
        int phased_per_sm = 0;
        WF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&phased_per_sm, phased_kernel(r->opaque, r->textured),
                                                              int(r->persistent_block_size), 0));
        if (per_sm <= 0 || phased_per_sm <= 0) return fail(WF_ERR_UNSUPPORTED, "the persistent kernel cannot be resident");
        // the largest grids; persistent_grid picks each launch's
        r->persistent_blocks = uint32_t(per_sm) * uint32_t(r->sm_count);
        r->phased_blocks = uint32_t(phased_per_sm) * uint32_t(r->sm_count);
        r->chunk = c.chunk ? std::max(1u, c.chunk / 32) : 1u;
    }
    if (c.caustics && photon_source) {
        r->params.photons = photon_source->params.photons;
        r->photons_emitted = photon_source->photons_emitted;
        r->photons_stored = photon_source->photons_stored;
    } else if (c.caustics) {
        if (wf_status e = build_photon_map(rr)) return e;
    }
    if (c.mode != WF_MODE_PERSISTENT) {
        WF_CUDA(cudaStreamCreateWithFlags(&r->side, cudaStreamNonBlocking));
        WF_CUDA(cudaEventCreateWithFlags(&r->fork_event, cudaEventDisableTiming));
        WF_CUDA(cudaEventCreateWithFlags(&r->join_event, cudaEventDisableTiming));
    }
    if (c.mode == WF_MODE_GRAPH || c.mode == WF_MODE_STREAM) {
        wf_status e = c.mode == WF_MODE_GRAPH ? capture_graph(rr) : capture_stream_graph(rr);
        if (e != WF_OK) {
            abandon_capture(r->stream);
            return e;
        }
    }
    WF_CUDA(cudaStreamSynchronize(r->stream));
    *out = r.release();
    return WF_OK;
}
}  // namespace

wf_status renderer_create(const wf_scene* scene, const wf_camera* camera, const wf_render_config* cfg, void* stream,
                          wf_renderer** out) {
    wf_renderer* r = nullptr;
    if (wf_status e = renderer_create_impl(scene, camera, cfg, stream, &r, nullptr, nullptr)) return e;
    if (cfg->mode == WF_MODE_GRAPH && cfg->concurrent_tiles != 1) {
        wf_render_config twin_config = *cfg;
        twin_config.concurrent_tiles = 1;
        wf_renderer* twin = nullptr;
        wf_status e = renderer_create_impl(scene, camera, &twin_config, nullptr, &twin, r->framebuffer, r);
        cudaError_t ce = cudaSuccess;
        if (e == WF_OK) {
            r->twin = twin;
            ce = cudaEventCreateWithFlags(&r->twin_fork, cudaEventDisableTiming);
            if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&r->twin_join, cudaEventDisableTiming);
        }
        if (e != WF_OK || ce != cudaSuccess) {
            renderer_destroy(r);
            return e != WF_OK ? e : cuda_fail(ce, "cudaEventCreateWithFlags");
        }
    }
    *out = r;
    return WF_OK;
}

wf_status renderer_destroy(wf_renderer* r) {
    if (!r) return WF_OK;
    if (r->twin) renderer_destroy(r->twin);
    if (r->twin_fork) cudaEventDestroy(r->twin_fork);
    if (r->twin_join) cudaEventDestroy(r->twin_join);
    if (r->copy_stream) {
        cudaStreamSynchronize(r->copy_stream);
        cudaStreamDestroy(r->copy_stream);
    }
    for (int k = 0; k < 2; ++k) {
        if (r->snapshot_ready[k]) cudaEventDestroy(r->snapshot_ready[k]);
        if (r->copy_done[k]) cudaEventDestroy(r->copy_done[k]);
    }
    if (r->stream) cudaStreamSynchronize(r->stream);
    for (auto& slot : r->slots) {
        if (slot->writer.joinable()) slot->writer.join();
        if (slot->pixels) cudaFreeHost(slot->pixels);
        if (slot->copied) cudaEventDestroy(slot->copied);
    }
    if (r->graph_exec) cudaGraphExecDestroy(r->graph_exec);
    if (r->graph) cudaGraphDestroy(r->graph);
    if (r->fork_event) cudaEventDestroy(r->fork_event);
    if (r->join_event) cudaEventDestroy(r->join_event);
    if (r->side) cudaStreamDestroy(r->side);
    for (void* p : r->allocations) cudaFree(p);
    if (r->own_stream) cudaStreamDestroy(r->stream);
    delete r;
    return WF_OK;
}

wf_status renderer_render(wf_renderer* r, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_start,
                          uint32_t sample_count, uint32_t clear) {
    const wf_render_config& c = r->config;
    if (w == 0 || h == 0 || x >= c.width || y >= c.height || w > c.width - x || h > c.height - y ||
        uint64_t(w) * h > r->tile_capacity)
        return fail(WF_ERR_INVALID_ARG, "Render task tile is outside the prepared renderer bounds");
    if (sample_count == 0) return fail(WF_ERR_INVALID_ARG, "Render task sample range is empty");
    if (clear) {
        WF_CUDA(cudaMemset2DAsync(r->framebuffer + (size_t(y) * c.width + x) * 3, size_t(c.width) * 12, 0,
                                  size_t(w) * 12, h, r->stream));
    }
    WF_CUDA(cudaMemcpyAsync(&r->counters->sample_index, &sample_start, sizeof(uint32_t), cudaMemcpyHostToDevice,
                            r->stream));
    if (r->twin && h >= 2) {
        // the top rows on this renderer, the bottom rows on the twin's stream
        wf_renderer* t = r->twin;
        uint32_t top = (h + 1) / 2;
        WF_CUDA(cudaEventRecord(r->twin_fork, r->stream));
        WF_CUDA(cudaStreamWaitEvent(t->stream, r->twin_fork, 0));
        WF_CUDA(cudaMemcpyAsync(&t->counters->sample_index, &sample_start, sizeof(uint32_t), cudaMemcpyHostToDevice,
                                t->stream));
        TileDev a{x, y, w, top, 1}, b{x, y + top, w, h - top, 1};
        r->last_tile_parts = 3;
        for (uint32_t s = 0; s < sample_count; s += a.samples) {
            a.samples = b.samples = std::min(r->wave, sample_count - s);
            if (wf_status e = launch_tile(r, a)) return e;
            if (wf_status e = launch_tile(t, b)) return e;
        }
        WF_CUDA(cudaEventRecord(r->twin_join, t->stream));
        WF_CUDA(cudaStreamWaitEvent(r->stream, r->twin_join, 0));
        // both sample indices end at sample_start + sample_count
        return WF_OK;
    }
    TileDev tile{x, y, w, h, 1};
    if (c.mode == WF_MODE_STREAM) {
        tile.samples = sample_count;
        return launch_tile(r, tile);
    }
    for (uint32_t s = 0; s < sample_count; s += tile.samples) {
        tile.samples = std::min(r->wave, sample_count - s);
        if (wf_status e = launch_tile(r, tile)) return e;
    }
    r->last_tile_parts = 1;
    if (r->twin) {  // a one-row task ran here alone: the twin's sample index follows
        uint32_t end = sample_start + sample_count;
        WF_CUDA(cudaEventRecord(r->twin_fork, r->stream));
        WF_CUDA(cudaStreamWaitEvent(r->twin->stream, r->twin_fork, 0));
        WF_CUDA(cudaMemcpyAsync(&r->twin->counters->sample_index, &end, sizeof(uint32_t), cudaMemcpyHostToDevice,
                                r->twin->stream));
        WF_CUDA(cudaStreamSynchronize(r->twin->stream));
    }
    return WF_OK;
}

wf_status renderer_render_frame(wf_renderer* r, uint32_t sample_count) {
    const wf_render_config& c = r->config;
    uint32_t tw = c.tile_width && c.tile_height ? c.tile_width : c.width;
    uint32_t th = c.tile_width && c.tile_height ? c.tile_height : c.height;
    std::vector<TileDev> tiles;
    for (uint32_t y = 0; y < c.height; y += th)
        for (uint32_t x = 0; x < c.width; x += tw)
            tiles.push_back(TileDev{x, y, std::min(tw, c.width - x), std::min(th, c.height - y), 0});
    if (c.mode == WF_MODE_STREAM) {
        // Tile-major: each tile takes the whole sample range in one launch;
        // every pixel belongs to one tile, so its sample order is unchanged.
        for (size_t t = 0; t < tiles.size(); ++t) {
            TileDev tile = tiles[t];
            tile.samples = sample_count;
            tile.advance_sample = t + 1 == tiles.size() ? 1u : 0u;
            if (wf_status e = launch_tile(r, tile)) return e;
        }
        return WF_OK;
    }
    if (r->twin) {
        // Rows of a single frame tile, or whole tiles alternately, go to the
        // two wavefronts; each advances its own sample index once per sample.
        wf_renderer* twin = r->twin;
        std::vector<TileDev> mine, theirs;
        if (tiles.size() == 1 && tiles[0].height >= 2) {
            TileDev a = tiles[0], b = tiles[0];
            a.height = (tiles[0].height + 1) / 2;
            b.y = tiles[0].y + a.height;
            b.height = tiles[0].height - a.height;
            mine.push_back(a);
            theirs.push_back(b);
        } else {
            for (size_t t = 0; t < tiles.size(); ++t) (t % 2 ? theirs : mine).push_back(tiles[t]);
        }
        // queue counts report the frame's last tile: both halves, or the part that rendered it
        r->last_tile_parts = theirs.empty() ? 1u : (mine.size() == 1 && theirs.size() == 1 && tiles.size() == 1)
                                                        ? 3u
                                                        : (tiles.size() % 2 ? 1u : 2u);
        WF_CUDA(cudaEventRecord(r->twin_fork, r->stream));
        WF_CUDA(cudaStreamWaitEvent(twin->stream, r->twin_fork, 0));
        for (uint32_t s = 0, k = 0; s < sample_count; s += k) {
            k = std::min(r->wave, sample_count - s);
            for (int part = 0; part < 2; ++part) {
                std::vector<TileDev>& list = part ? theirs : mine;
                for (size_t t = 0; t < list.size(); ++t) {
                    TileDev tile = list[t];
                    tile.advance_sample = t + 1 == list.size() ? 1u : 0u;
                    tile.samples = k;
                    if (wf_status e = launch_tile(part ? twin : r, tile)) return e;
                }
                if (list.empty() && part) {  // a single one-row frame: keep the twin's sample index in step
                    TileDev idle{0, 0, 0, 0, 1};
                    idle.samples = k;
                    WF_CUDA(cudaMemcpyAsync(twin->tile, &idle, sizeof(TileDev), cudaMemcpyHostToDevice, twin->stream));
                    k_advance<<<1, 1, 0, twin->stream>>>(twin->counters, twin->tile);
                    WF_CUDA(cudaGetLastError());
                }
            }
        }
        WF_CUDA(cudaEventRecord(r->twin_join, twin->stream));
        WF_CUDA(cudaStreamWaitEvent(r->stream, r->twin_join, 0));
        return WF_OK;
    }
    for (uint32_t s = 0, k = 0; s < sample_count; s += k) {
        k = std::min(r->wave, sample_count - s);
        for (size_t t = 0; t < tiles.size(); ++t) {
            TileDev tile = tiles[t];
            tile.advance_sample = t + 1 == tiles.size() ? 1u : 0u;
            tile.samples = k;
            if (wf_status e = launch_tile(r, tile)) return e;
        }
    }
    return WF_OK;
}

namespace {
std::vector<TileDev> frame_tiles(const wf_render_config& c) {
    uint32_t tw = c.tile_width && c.tile_height ? c.tile_width : c.width;
    uint32_t th = c.tile_width && c.tile_height ? c.tile_height : c.height;
    std::vector<TileDev> tiles;
    for (uint32_t y = 0; y < c.height; y += th)
        for (uint32_t x = 0; x < c.width; x += tw)
            tiles.push_back(TileDev{x, y, std::min(tw, c.width - x), std::min(th, c.height - y), 0});
    tiles.back().advance_sample = 1;
    return tiles;
}
}  // namespace

wf_status renderer_profile(wf_renderer* r, wf_kernel_profile* out) {
    std::memset(out, 0, sizeof(*out));
    std::vector<TileDev> tiles = frame_tiles(r->config);
    cudaStream_t st = r->stream;
    cudaEvent_t e0, e1;
    WF_CUDA(cudaEventCreate(&e0));
    WF_CUDA(cudaEventCreate(&e1));
    float last_ms = 0.0f;
    auto timed = [&](int kind, auto&& launch) -> wf_status {
        WF_CUDA(cudaEventRecord(e0, st));
        launch();
        WF_CUDA(cudaGetLastError());
        WF_CUDA(cudaEventRecord(e1, st));
        WF_CUDA(cudaEventSynchronize(e1));
        last_ms = 0.0f;
        WF_CUDA(cudaEventElapsedTime(&last_ms, e0, e1));
        out->milliseconds[kind] += last_ms;
        out->launches[kind] += 1;
        return WF_OK;
    };
    // Every read goes through the renderer stream: it may be a non-blocking
    // stream, which a plain cudaMemcpy on the legacy stream does not wait for.
    auto read_back = [&](void* dst, const void* src, size_t bytes) -> wf_status {
        WF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
        WF_CUDA(cudaStreamSynchronize(st));
        return WF_OK;
    };
    unsigned long long before[2], after[2];
    if (wf_status e = read_back(before, &r->counters->extension_rays, sizeof(before))) return e;
    if (r->config.mode == WF_MODE_PERSISTENT) {
        for (const TileDev& tile : tiles) {
            WF_CUDA(cudaMemcpyAsync(r->tile, &tile, sizeof(TileDev), cudaMemcpyHostToDevice, st));
            cudaError_t launch_error = cudaSuccess;
            if (wf_status e = timed(WF_KERNEL_PERSISTENT, [&] {
                    launch_error = launch_persistent(r, st, uint64_t(tile.width) * tile.height);
                }))
                return e;
            WF_CUDA(launch_error);
            k_advance<<<1, 1, 0, st>>>(r->counters, r->tile);
        }
    } else {
        if (!r->tally) WF_CUDA(alloc(r, &r->tally, 2));
        const DeviceScene& s = r->scene->view;
        uint32_t cap = r->capacity;
        for (int pass = 0; pass < 2; ++pass) {
            bool count = pass == 1;
            if (count) WF_CUDA(cudaMemsetAsync(r->tally, 0, 2 * sizeof(TallyTotals), st));
            for (TileDev tile : tiles) {
                tile.samples = r->wave;  // the graph's launches: one wave of samples
                WF_CUDA(cudaMemcpyAsync(r->tile, &tile, sizeof(TileDev), cudaMemcpyHostToDevice, st));
                auto raygen = [&] {
                    k_raygen<<<grid_for(r, cap, 256), 256, 0, st>>>(r->params, r->tile, r->counters, r->paths,
                                                                     r->queue[0], cap);
                };
                if (count) raygen(); else if (wf_status e = timed(WF_KERNEL_RAYGEN, raygen)) return e;
                for (uint32_t b = 0; b < r->config.max_depth; ++b) {
                    uint32_t cur = b & 1, nxt = cur ^ 1;
                    uint32_t* cur_count = &r->counters->queue_count[cur];
                    uint32_t* next_count = &r->counters->queue_count[nxt];
                    auto trace = [&] {
                        if (count && b == 0)
                            launch_trace<CountTally, false>(r, grid(r, 5, cap, r->block_camera), r->block_camera, st, 
                                s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, b,
                                r->tally, r->refill, nullptr, nullptr);
                        else if (count)
                            launch_trace<CountTally, true>(r, grid(r, 0, cap, r->block_trace), r->block_trace, st, 
                                s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, b,
                                r->tally, r->refill, nullptr, nullptr);
                        else if (b == 0)
                            launch_trace<NoTally, false>(r, grid(r, 5, cap, r->block_camera), r->block_camera, st, 
                                s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, b,
                                nullptr, r->refill, nullptr, nullptr);
                        else
                            launch_trace<NoTally, true>(r, grid(r, 0, cap, r->block_trace), r->block_trace, st, 
                                s, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->counters, b,
                                nullptr, r->refill, nullptr, nullptr);
                    };
                    auto shade = [&] {  // with the category sort it feeds on
                        if (r->sort_shading) {
                            k_classify<<<grid(r, 3, cap, 256), 256, 0, st>>>(s, cur_count, r->hit_a, r->hit_inst,
                                                                              r->shade_key, r->counters);
                            k_scatter<<<grid(r, 3, cap, 256), 256, 0, st>>>(cur_count, r->shade_key,
                                                                             r->shade_order, r->counters);
                        }
                        launch_shade(r, grid(r, 1, cap, r->block_shade), r->block_shade, st, 
                            s, r->params, r->paths, r->queue[cur], cur_count, r->hit_a, r->hit_inst, r->terms,
                            r->shade_out, r->shadow_origin, r->shadow_dir, r->shadow_capacity, r->counters,
                            next_count, r->gathers, r->sort_shading ? r->shade_order : nullptr);
                    };
                    auto gather = [&] {
                        k_gather<<<grid(r, 4, cap, r->block_gather), r->block_gather, 0, st>>>(r->params, r->gathers,
                                                                                               r->terms, r->counters);
                        k_gather_dense<<<grid(r, 4, cap, r->block_gather), r->block_gather, 0, st>>>(
                            r->params, r->gathers, r->terms, r->counters);
                    };
                    bool gathers = r->params.photons.enabled != 0;
                    auto shadow = [&] {
                        if (count)
                            launch_shadow<CountTally>(r, grid(r, 2, r->shadow_capacity, r->block_trace), r->block_trace, st, s, r->shadow_origin, r->shadow_dir, r->shadow_result,
                                                            r->counters, r->shadow_capacity, r->tally + 1, r->refill);
                        else
                            launch_shadow<NoTally>(r, grid(r, 2, r->shadow_capacity, r->block_trace), r->block_trace, st, s, r->shadow_origin, r->shadow_dir, r->shadow_result,
                                                      r->counters, r->shadow_capacity, nullptr, r->refill);
                    };
                    auto finalize = [&] {
                        k_finalize<false><<<grid(r, 3, cap, r->block_finalize), r->block_finalize, 0, st>>>(
                            r->paths, r->queue[cur], cur_count, r->terms, r->shade_out, r->shadow_result,
                            r->queue[nxt], next_count, cap, r->framebuffer, &r->counters->work_trace, r->params,
                            r->tile, r->counters);
                    };
                    if (count) {
                        trace();
                        WF_CUDA(cudaGetLastError());
                        shade();
                        WF_CUDA(cudaGetLastError());
                        if (gathers) gather();
                        shadow();
                        WF_CUDA(cudaGetLastError());
                        finalize();
                        WF_CUDA(cudaGetLastError());
                    } else {
                        uint32_t pb = std::min<uint32_t>(b, WF_PROFILE_BOUNCES - 1);
                        const int kinds[5] = {WF_KERNEL_TRACE, WF_KERNEL_SHADE, WF_KERNEL_SHADOW, WF_KERNEL_FINALIZE,
                                              WF_KERNEL_GATHER};
                        const int order[5] = {0, 1, 4, 2, 3};  // trace, shade, gather, shadow, finalize
                        for (int step = 0; step < 5; ++step) {
                            int k = order[step];
                            if (k == 4 && !gathers) continue;
                            wf_status e = k == 0   ? timed(kinds[k], trace)
                                          : k == 1 ? timed(kinds[k], shade)
                                          : k == 2 ? timed(kinds[k], shadow)
                                          : k == 3 ? timed(kinds[k], finalize)
                                                   : timed(kinds[k], gather);
                            if (e) return e;
                            out->bounce_milliseconds[k][pb] += last_ms;
                            if (k == 2) {  // after the shadow kernel: rays traced and shadow rays of this bounce
                                uint32_t rays[2];
                                if (wf_status e2 = read_back(&rays[0], cur_count, sizeof(uint32_t))) return e2;
                                if (wf_status e2 = read_back(&rays[1], &r->counters->shadow_count, sizeof(uint32_t)))
                                    return e2;
                                out->bounce_extension_rays[pb] += rays[0];
                                out->bounce_shadow_rays[pb] += std::min(rays[1], r->shadow_capacity);
                            }
                        }
                    }
                }
                if (tile.samples > 1)
                    k_accumulate_wave<<<grid_for(r, r->tile_capacity, 256), 256, 0, st>>>(r->paths, r->tile,
                                                                                            r->framebuffer,
                                                                                            r->counters);
                k_advance<<<1, 1, 0, st>>>(r->counters, r->tile);
            }
            if (!count)
                if (wf_status e = read_back(after, &r->counters->extension_rays, sizeof(after))) return e;
        }
        TallyTotals t[2];
        if (wf_status e = read_back(t, r->tally, sizeof(t))) return e;
        out->closest_nodes = t[0].v[0];
        out->closest_triangles = t[0].v[1];
        out->closest_spheres = t[0].v[2];
        out->closest_instances = t[0].v[3];
        out->any_nodes = t[1].v[0];
        out->any_triangles = t[1].v[1];
        out->any_spheres = t[1].v[2];
        out->any_instances = t[1].v[3];
    }
    if (r->config.mode == WF_MODE_PERSISTENT)
        if (wf_status e = read_back(after, &r->counters->extension_rays, sizeof(after))) return e;
    out->extension_rays = after[0] - before[0];
    out->shadow_rays = after[1] - before[1];
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    WF_CUDA(cudaStreamSynchronize(st));
    r->last_tile_parts = 1;
    if (r->twin) {  // the pass ran on this renderer alone: bring the twin's sample index along
        uint32_t index = 0;
        if (wf_status e = read_back(&index, &r->counters->sample_index, sizeof(index))) return e;
        WF_CUDA(cudaMemcpyAsync(&r->twin->counters->sample_index, &index, sizeof(index), cudaMemcpyHostToDevice,
                                r->twin->stream));
        WF_CUDA(cudaStreamSynchronize(r->twin->stream));
    }
    return WF_OK;
}

wf_status trace_closest_batch(const wf_scene* scene, const wf_ray* rays, uint32_t count, wf_hit* hits,
                              cudaStream_t stream) {
    if (count == 0) return WF_OK;
    k_trace_batch<<<(count + 127) / 128, 128, 0, stream>>>(scene->view, rays, count, hits);
    WF_CUDA(cudaGetLastError());
    return WF_OK;
}

wf_status trace_any_batch(const wf_scene* scene, const wf_ray* rays, const float* max_distance, uint32_t count,
                          uint8_t* occluded, cudaStream_t stream) {
    if (count == 0) return WF_OK;
    k_any_batch<<<(count + 127) / 128, 128, 0, stream>>>(scene->view, rays, max_distance, count, occluded);
    WF_CUDA(cudaGetLastError());
    return WF_OK;
}

}  // namespace wf

// ---------------------------------------------------------------------------
// wf_render_tile_static: the persistent-mode tile render with its working
// memory in a fixed device array instead of cudaMalloc'd buffers.
//
// Some hosts cannot allocate device memory at render time: a caller running
// inside another framework's memory pool, under a strict memory budget
// that was fixed at start-up, or from a context where cudaMalloc would
// synchronize the device.  They still own their inputs (the scene) and
// outputs (the framebuffer); this entry point needs nothing else.  The cost
// is a file-scope array that every GPU loading this library holds until the
// process exits, and a cap on the tile size.
namespace wf {
namespace {

constexpr uint32_t kStaticMaxPixels = 65536;  // one 256 x 256 tile

// Scratch layout (each part 256-byte aligned): counters, tile, path state
// (origin, direction, throughput, radiance as float4; info as uint4; RNG
// state as u64) and the two index queues, kStaticMaxPixels slots each.
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kStaticCountersOffset = 0;
constexpr size_t kStaticTileOffset = align256(kStaticCountersOffset + sizeof(Counters));
constexpr size_t kStaticPathOffset = align256(kStaticTileOffset + sizeof(TileDev));
constexpr size_t kStaticFloat4Bytes = size_t(kStaticMaxPixels) * sizeof(float4);
constexpr size_t kStaticInfoOffset = kStaticPathOffset + 4 * kStaticFloat4Bytes;
constexpr size_t kStaticRngOffset = align256(kStaticInfoOffset + size_t(kStaticMaxPixels) * sizeof(uint4));
constexpr size_t kStaticQueueOffset = align256(kStaticRngOffset + size_t(kStaticMaxPixels) * sizeof(uint64_t));
constexpr size_t kStaticBytes = align256(kStaticQueueOffset + 2 * size_t(kStaticMaxPixels) * sizeof(uint32_t));

// 6.3 MB per device.  Host code must not use this name as a device address:
// the host sees a stand-in object; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mutex;
unsigned char* g_static_base[kStaticMaxDevices] = {};
unsigned long long g_static_context[kStaticMaxDevices] = {};  // context the address belongs to
uint32_t g_static_resident[kStaticMaxDevices][3] = {};  // per persistent-kernel variant

// Unique id of the calling thread's current context (cuCtxGetId), or 0 when
// none is current.  A device whose context is re-created (cudaDeviceReset,
// then any runtime call) loads the module again, and the array may move: the
// id changes with it, so the set-up runs again for the new context.  The
// driver functions come from cudaGetDriverEntryPoint, so the library needs no
// link against libcuda.
cudaError_t current_context_id(unsigned long long& id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    id = 0;
    if (!get_current || !get_id) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa{}, qb{};
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa);
        if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb);
        if (e != cudaSuccess) return e;
        if (qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
            return cudaErrorNotSupported;
        get_current = reinterpret_cast<GetCurrent>(a);
        get_id = reinterpret_cast<GetId>(b);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return cudaErrorContextIsDestroyed;
    if (!ctx) return cudaSuccess;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return cudaErrorContextIsDestroyed;
    return cudaSuccess;
}

// Zeroes the counters at the start of a call (the array keeps the previous
// call's contents) and writes the tile and the first sample index.
__global__ void k_static_prepare(Counters* c, TileDev* tile_out, TileDev tile, uint32_t sample_start) {
    uint32_t* words = reinterpret_cast<uint32_t*>(c);
    for (size_t i = threadIdx.x; i < sizeof(Counters) / sizeof(uint32_t); i += blockDim.x) words[i] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        c->sample_index = sample_start;
        *tile_out = tile;
    }
}

// Per-sample reset of the persistent kernel's queue counters and barrier
// arrival count (what launch_tile clears with memsets).
__global__ void k_static_sample_reset(Counters* c) {
    for (uint32_t i = threadIdx.x; i < 2 * (kMaxBounces + 1); i += blockDim.x) c->persistent_count[i] = 0;
    if (threadIdx.x == 0) c->barrier_count = 0;
}

}  // namespace
}  // namespace wf

extern "C" wf_status wf_render_tile_static(const wf_scene* scene, const wf_camera* camera,
                                          const wf_render_config* config, uint32_t x, uint32_t y, uint32_t width,
                                          uint32_t height, uint32_t sample_start, uint32_t sample_count,
                                          float* framebuffer, void* stream) {
    using namespace wf;
    if (!scene || !camera || !config || !framebuffer) return fail(WF_ERR_INVALID_ARG, "null argument");
    const wf_render_config& c = *config;
    if (wf_status e = check_render_config(scene, c)) return e;
    if (c.caustics)
        return fail(WF_ERR_UNSUPPORTED, "wf_render_tile_static does not build photon maps (caustics must be 0)");
    if (width == 0 || height == 0 || x >= c.width || y >= c.height || width > c.width - x || height > c.height - y)
        return fail(WF_ERR_INVALID_ARG, "Render task tile is outside the framebuffer");
    if (uint64_t(width) * height > kStaticMaxPixels)
        return fail(WF_ERR_CAPACITY, "wf_render_tile_static renders at most %u pixels per call (tile is %ux%u)",
                    kStaticMaxPixels, width, height);
    if (sample_count == 0) return fail(WF_ERR_INVALID_ARG, "Render task sample range is empty");
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Once per device: the device address of the scratch array and the
    // persistent kernel's resident grid.
    int device = 0;
    WF_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= kStaticMaxDevices) return fail(WF_ERR_UNSUPPORTED, "device index %d", device);
    unsigned char* base = nullptr;
    uint32_t resident = 0;
    const bool opaque = !scene->alpha_textures;
    const void* kernel = persistent_kernel(opaque, scene->textured);
    const int variant = !opaque ? 0 : (scene->textured ? 1 : 2);
    {
        std::lock_guard<std::mutex> lock(g_static_mutex);
        unsigned long long context = 0;
        WF_CUDA(current_context_id(context));
        if (!g_static_base[device] || context == 0 || context != g_static_context[device]) {
            // Set-up for this device's current context, with that device
            // current: the runtime binds its primary context here if no
            // context was current yet.
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
            WF_CUDA(current_context_id(context));
            int cooperative = 0;
            WF_CUDA(cudaDeviceGetAttribute(&cooperative, cudaDevAttrCooperativeLaunch, device));
            if (!cooperative) return fail(WF_ERR_UNSUPPORTED, "device does not support cooperative launches");
            g_static_base[device] = static_cast<unsigned char*>(p);
            g_static_context[device] = context;
        }
        if (!g_static_resident[device][variant]) {
            int sms = 0, per_sm = 0;
            WF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
            WF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0));
            if (per_sm <= 0) return fail(WF_ERR_UNSUPPORTED, "the persistent kernel cannot be resident");
            g_static_resident[device][variant] = uint32_t(per_sm) * uint32_t(sms);
        }
        base = g_static_base[device];
        resident = g_static_resident[device][variant];
    }

    // The same parameters renderer_create derives for a persistent renderer.
    RenderParams rp{};
    rp.width = c.width;
    rp.height = c.height;
    rp.max_depth = c.max_depth;
    rp.rr_start = c.rr_start_depth;
    rp.rng = c.rng;
    rp.debug = c.debug;
    rp.clamp = c.indirect_clamp;
    rp.gather_radius = c.gather_radius;
    rp.camera.position = V3{camera->position[0], camera->position[1], camera->position[2]};
    rp.camera.forward = V3{camera->forward[0], camera->forward[1], camera->forward[2]};
    rp.camera.right = V3{camera->right[0], camera->right[1], camera->right[2]};
    rp.camera.up = V3{camera->up[0], camera->up[1], camera->up[2]};
    rp.camera.aspect_ratio = camera->aspect_ratio;
    rp.camera.tan_half_fov = wfm::tanf(camera->vertical_fov * 0.5f);
    rp.photons = PhotonGridView{};
    int sms = 0;
    WF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    uint32_t blocks = persistent_grid(c.persistent_blocks, resident, uint32_t(sms), uint64_t(width) * height);
    uint32_t chunk = c.chunk ? std::max(1u, c.chunk / 32) : 1u;

    Counters* counters = reinterpret_cast<Counters*>(base + kStaticCountersOffset);
    TileDev* tile_dev = reinterpret_cast<TileDev*>(base + kStaticTileOffset);
    PathSoA ps{};
    ps.origin = reinterpret_cast<float4*>(base + kStaticPathOffset);
    ps.direction = ps.origin + kStaticMaxPixels;
    ps.throughput = ps.direction + kStaticMaxPixels;
    ps.radiance = ps.throughput + kStaticMaxPixels;
    ps.info = reinterpret_cast<uint4*>(base + kStaticInfoOffset);
    ps.rng = reinterpret_cast<unsigned long long*>(base + kStaticRngOffset);
    ps.slot_sample = nullptr;
    ps.wait = nullptr;
    uint32_t* q0 = reinterpret_cast<uint32_t*>(base + kStaticQueueOffset);
    uint32_t* q1 = q0 + kStaticMaxPixels;

    TileDev tile{x, y, width, height, 1};
    k_static_prepare<<<1, 256, 0, st>>>(counters, tile_dev, tile, sample_start);
    WF_CUDA(cudaGetLastError());
    DeviceScene s = scene->view;
    const TileDev* tp = tile_dev;
    uint32_t cap = kStaticMaxPixels;
    void* args[] = {&s, &rp, &tp, &counters, &ps, &q0, &q1, &cap, &framebuffer, &chunk};
    for (uint32_t i = 0; i < sample_count; ++i) {
        k_static_sample_reset<<<1, 128, 0, st>>>(counters);
        WF_CUDA(cudaLaunchCooperativeKernel(kernel, dim3(blocks), dim3(128), args, 0,
                                            st));
        k_advance<<<1, 1, 0, st>>>(counters, tile_dev);
        WF_CUDA(cudaGetLastError());
    }
    uint32_t error = 0;
    WF_CUDA(cudaMemcpyAsync(&error, &counters->error, sizeof(error), cudaMemcpyDeviceToHost, st));
    WF_CUDA(cudaStreamSynchronize(st));
    if (error) return fail(WF_ERR_TIMEOUT, "persistent kernel grid barrier timed out");
    return WF_OK;
}
