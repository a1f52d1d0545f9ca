// Job batch: many independent renders (own scene, camera, resolution, depth,
// sample range) in one captured CUDA graph.
//
// Work is a list of path units, one per (job, sample, pixel), job by job
// and, within a job, sample by sample in pixel order.  A pool of path slots
// runs the wavefront stages of the single-scene renderer (lane-refill
// closest hit, shading with deferred shadow rays, lane-refill occlusion,
// ordered term accumulation and compaction) inside a device-side WHILE
// loop; a slot whose path ends stores the path's radiance by unit and takes
// the next unit from a device counter, so the pool stays full until the
// last paths of the pass.  After each pass, k_batch_accumulate adds every
// pixel's radiances to its job's framebuffer in sample order, the order in
// which a per-job wf_render adds them: the framebuffers are bit-identical.
// Jobs with few pixels or few samples pay no per-launch and per-bounce
// overheads of their own, and no pixel's samples form a serial chain.  A
// batch of more units than one pass holds (the radiance buffer's size) runs
// as several passes in unit order.
#include "wf_wavefront.cuh"
#include "wf_lane_traverse.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

namespace wf {

struct BatchJob {
    DeviceScene scene;
    RenderParams rp;
    unsigned long long fb_offset;  // first float of the job framebuffer
    uint32_t unit_begin;           // first unit of the job: unit_begin + k * pixels + q is sample k of pixel q
    uint32_t pixels;
    uint32_t sample_start, sample_count;
};

// Device view of a batch (kernel parameter).
struct BatchView {
    const BatchJob* jobs;
    const uint32_t* job_order;    // jobs in unit order
    const uint32_t* order_units;  // first unit of each job in unit order (ascending)
    const uint32_t* order_pixels; // first pixel of each job in unit order, over all jobs' pixels
    uint32_t job_count;
    uint32_t units;               // path units of the whole batch
    uint32_t pixels;              // pixels of all jobs
    uint32_t* slot_job;
    uint32_t* slot_unit;
    float4* unit_radiance;        // radiance of each unit of the current pass, by unit - pass_begin
    float* framebuffer;
};

}  // namespace wf

struct wf_batch {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool opaque = true;     // no job's scene has alpha-textured materials: the Opaque<> trace and shadow kernels
    bool textured = false;  // some job's scene has textured materials: k_batch_shade<true>
    int device = 0, sm_count = 148;
    std::vector<void*> allocations;
    std::vector<wf_batch_job> jobs;
    std::vector<unsigned long long> fb_offsets;
    size_t fb_floats = 0;
    wf::BatchView view{};
    wf::BatchJob* jobs_dev = nullptr;
    uint32_t* order_dev = nullptr;  // job_order, order_units, order_pixels
    wf::PathSoA paths{};
    uint32_t* queue[2] = {nullptr, nullptr};
    float4* hit_a = nullptr;
    uint32_t* hit_inst = nullptr;
    float4* terms = nullptr;
    int4* shade_out = nullptr;
    float4* shadow_origin = nullptr;
    float4* shadow_dir = nullptr;
    uint8_t* shadow_result = nullptr;
    uint32_t shadow_capacity = 0;
    wf::Counters* counters = nullptr;
    uint32_t capacity = 0, units = 0, pass_units = 0, block = 128, refill = 8, max_depth = 1;
    uint32_t grid_resident[4] = {0, 0, 0, 0};
    unsigned long long total_paths = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace wf {
namespace {

#define WF_BATCH_CUDA(call)                                       \
    do {                                                          \
        cudaError_t wf_e_ = (call);                               \
        if (wf_e_ != cudaSuccess) return cuda_fail(wf_e_, #call); \
    } while (0)

// Position (in unit order) of the largest first value <= v in ascending `first`.
WF_DEV uint32_t batch_position(const uint32_t* first, uint32_t count, uint32_t v) {
    uint32_t lo = 0, hi = count;  // first[lo] <= v < first[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (first[mid] <= v) lo = mid; else hi = mid;
    }
    return lo;
}

// Starts `unit` (a sample of one pixel of one job) in `slot`.
WF_DEV void batch_start(const BatchView& b, const PathSoA& ps, uint32_t slot, uint32_t unit) {
    uint32_t job = b.job_order[batch_position(b.order_units, b.job_count, unit)];
    const BatchJob& J = b.jobs[job];
    uint32_t local = unit - J.unit_begin;
    uint32_t k = local / J.pixels;
    TileDev tile{0, 0, J.rp.width, J.rp.height, 0};
    Path path;
    init_path(J.rp, tile, J.sample_start + k, local - k * J.pixels, path);
    store_path(ps, slot, path);
    ps.radiance[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    b.slot_job[slot] = job;
    b.slot_unit[slot] = unit;
}

__global__ void k_batch_raygen(BatchView b, Counters* c, PathSoA ps, uint32_t* queue, uint32_t capacity) {
    count_launch(c);
    uint32_t begin = c->pass_begin;
    uint32_t n = min(capacity, c->pass_end - begin);
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        c->queue_count[0] = n;
        c->next_unit = begin + n;
        c->paths += c->pass_end - begin;
        c->work_trace = 0;
        c->stream_iterations = 0;
    }
    for (uint32_t slot = gid; slot < n; slot += gridDim.x * blockDim.x) {
        batch_start(b, ps, slot, begin + slot);
        queue[slot] = slot;
    }
}

// After a pass: every pixel of every job adds the radiances of its samples
// in the pass to the job framebuffer, in sample order.
__global__ void k_batch_accumulate(BatchView b, const Counters* c) {
    uint32_t begin = c->pass_begin, end = c->pass_end;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < b.pixels; t += gridDim.x * blockDim.x) {
        uint32_t pos = batch_position(b.order_pixels, b.job_count, t);
        const BatchJob& J = b.jobs[b.job_order[pos]];
        uint32_t q = t - b.order_pixels[pos];
        uint64_t first = J.unit_begin, last = first + uint64_t(J.pixels) * J.sample_count;
        if (last <= begin || first >= end) continue;
        float* f = b.framebuffer + J.fb_offset + 3 * size_t(q);
        float r = f[0], g = f[1], bl = f[2];
        for (uint32_t k = 0; k < J.sample_count; ++k) {
            uint64_t unit = first + uint64_t(k) * J.pixels + q;
            if (unit < begin) continue;
            if (unit >= end) break;
            float4 rad = b.unit_radiance[unit - begin];
            r += rad.x;
            g += rad.y;
            bl += rad.z;
        }
        f[0] = r;
        f[1] = g;
        f[2] = bl;
    }
}

// At most 72 registers, as k_trace (7 CTAs of 128 per SM instead of 6).
template <typename Tally>
__global__ void __maxnreg__(72) k_batch_trace(BatchView b, PathSoA ps, const uint32_t* queue, const uint32_t* count, float4* hit_a,
                              uint32_t* hit_inst, Counters* c, uint32_t refill_at) {
    count_launch(c);
    uint32_t n = *count;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        c->shadow_count = 0;
        c->gather_count = 0;
        c->work_shade = 0;
        c->extension_rays += n;
    }
    Tally tally;
    ClosestLane L;
    L.stage = kStageDone;
    const DeviceScene* sp = nullptr;
    uint32_t i = 0;
    bool more = true;
    for (;;) {
        bool idle = L.stage == kStageDone;
        uint32_t slot = refill(&c->work_trace, n, idle, refill_at, more);
        if (slot != kInvalid) {
            i = slot;
            uint32_t p = queue[i];
            sp = &b.jobs[b.slot_job[p]].scene;
            float4 o = ps.origin[p], d = ps.direction[p];
            closest_begin(L, *sp, f4xyz(o), f4xyz(d), tally);
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
            closest_step(L, *sp, tally);
            if (L.stage == kStageDone) {
                hit_a[i] = make_float4(L.h.t, L.h.u, L.h.v, __uint_as_float(L.h.prim));
                hit_inst[i] = L.h.inst;
            }
        }
    }
}

template <bool kTextures>
__global__ void __launch_bounds__(128, 4) k_batch_shade(BatchView b, PathSoA ps, const uint32_t* queue,
                                                        const uint32_t* count, const float4* hit_a,
                                                        const uint32_t* hit_inst, float4* terms, int4* shade_out,
                                                        float4* shadow_origin, float4* shadow_dir,
                                                        uint32_t shadow_capacity, Counters* c, uint32_t* next_count) {
    count_launch(c);
    uint32_t n = *count;
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        *next_count = 0;
        c->work_shadow = 0;
        c->work_gather = 0;
    }
    uint32_t base;
    while (next_chunk(&c->work_shade, n, base)) {
        uint32_t i = base + (threadIdx.x & 31);
        if (i >= n) continue;
        uint32_t p = queue[i];
        uint32_t job = b.slot_job[p];
        const BatchJob& J = b.jobs[job];
        Path path = load_path(ps, p);
        float4 ha = hit_a[i];
        SurfaceHit sh;
        bool did_hit = finish_hit(J.scene, path.origin, path.direction, ha.x, ha.y, ha.z, __float_as_uint(ha.w),
                                  hit_inst[i], sh);
        DeferredSink sink{};
        sink.shadow_origin = shadow_origin;
        sink.shadow_dir = shadow_dir;
        sink.shadow_count = &c->shadow_count;
        sink.shadow_capacity = shadow_capacity;
        sink.terms = terms + size_t(i) * kMaxTerms;
        sink.owner = i;
        sink.tag = job;
        sink.nterms = 0;
        sink.kill = kUnconditional;
        sink.overflow = &c->overflow;
        bool alive = shade_path<DeferredSink, kTextures>(J.scene, J.rp, path, did_hit, sh, sink);
        if (sink.nterms > kMaxTerms) atomicOr(&c->overflow, 2u);
        store_path(ps, p, path);
        shade_out[i] = make_int4(min(sink.nterms, kMaxTerms), sink.kill, alive ? 1 : 0, 0);
    }
}

template <typename Tally>
__global__ void k_batch_shadow(BatchView b, const float4* shadow_origin, const float4* shadow_dir, uint8_t* result,
                               Counters* c, uint32_t capacity, uint32_t refill_at) {
    count_launch(c);
    uint32_t n = min(c->shadow_count, capacity);
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) c->shadow_rays += n;
    Tally tally;
    AnyLane L;
    L.stage = kStageDone;
    const DeviceScene* sp = nullptr;
    uint32_t j = 0;
    bool more = true;
    for (;;) {
        bool idle = L.stage == kStageDone;
        uint32_t slot = refill(&c->work_shadow, n, idle, refill_at, more);
        if (slot != kInvalid) {
            j = slot;
            float4 o = shadow_origin[j], d = shadow_dir[j];
            sp = &b.jobs[__float_as_uint(d.w)].scene;
            any_begin(L, *sp, f4xyz(o), f4xyz(d), o.w, tally);
            if (L.stage == kStageDone) result[j] = L.hit ? 1 : 0;
        }
        bool busy = L.stage != kStageDone;
        if (!__any_sync(0xffffffffu, busy)) {
            if (!more) break;
            continue;
        }
        if (busy) {
            any_step(L, *sp, tally);
            if (L.stage == kStageDone) result[j] = L.hit ? 1 : 0;
        }
    }
}

// Term accumulation, kill rule and compaction as in the single-scene
// finalize; an ended path stores its radiance by unit (k_batch_accumulate
// adds it after the pass), then its slot starts the pass's next unit.
__global__ void k_batch_finalize(BatchView b, PathSoA ps, const uint32_t* queue, const uint32_t* count,
                                 const float4* terms, const int4* shade_out, const uint8_t* shadow_result,
                                 uint32_t* next, uint32_t* next_count, uint32_t capacity, Counters* c) {
    count_launch(c);
    uint32_t n = *count;
    uint32_t lane = threadIdx.x & 31;
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) c->work_trace = 0;
    for (uint32_t base = warp * 32; base < n; base += warps * 32) {
        uint32_t i = base + lane;
        bool alive = false, need_unit = false;
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
            } else {
                b.unit_radiance[b.slot_unit[p] - c->pass_begin] = make_float4(rad.x, rad.y, rad.z, 0.0f);
                need_unit = true;
            }
        }
        unsigned want = __ballot_sync(0xffffffffu, need_unit);
        if (want) {
            uint32_t first = 0;
            if (lane == 0) first = atomicAdd(&c->next_unit, uint32_t(__popc(want)));
            first = __shfl_sync(0xffffffffu, first, 0);
            if (need_unit) {
                uint32_t unit = first + __popc(want & ((1u << lane) - 1u));
                if (unit < c->pass_end) {
                    batch_start(b, ps, p, unit);
                    alive = true;
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

// Loop condition with a hard bound (every slot runs at most
// units * max_depth bounces in a pass).
__global__ void k_batch_condition(cudaGraphConditionalHandle handle, Counters* c, unsigned long long bound) {
    count_launch(c);
    uint32_t it = ++c->stream_iterations;
    bool live = c->queue_count[0] > 0;
    if (live && it >= bound) {
        c->error = kErrorStreamBound;
        live = false;
    }
    cudaGraphSetConditional(handle, live ? 1u : 0u);
}

template <typename T>
cudaError_t batch_alloc(wf_batch* b, T** p, size_t count) {
    cudaError_t e = device_alloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(count, 1));
    if (e == cudaSuccess) b->allocations.push_back(*p);
    return e;
}

uint32_t batch_grid(const wf_batch* b, int kernel, uint32_t work, uint32_t block) {
    uint32_t g = std::max(1u, (work + block - 1) / block);
    return b->grid_resident[kernel] ? std::min(g, b->grid_resident[kernel]) : g;
}

template <typename K>
cudaError_t batch_resident(wf_batch* b, int kernel, K* fn, uint32_t block) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, int(block), 0);
    if (e == cudaSuccess) b->grid_resident[kernel] = uint32_t(std::max(per_sm, 1)) * uint32_t(b->sm_count);
    return e;
}

// Units per pass: the radiance buffer holds one float4 per unit of a pass
// (2 GB at this size); larger batches run as several passes.
constexpr uint64_t kBatchPassUnits = 1ull << 27;

// One run of the batch: for each pass, the pass's units go to the device,
// the graph renders them, and the pixels add their samples in order.
cudaError_t batch_run(wf_batch* b) {
    for (uint64_t begin = 0; begin < b->units; begin += b->pass_units) {
        uint32_t range[2] = {uint32_t(begin), uint32_t(std::min<uint64_t>(b->units, begin + b->pass_units))};
        cudaError_t e = cudaMemcpyAsync(&b->counters->pass_begin, range, sizeof(range), cudaMemcpyHostToDevice,
                                        b->stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, b->stream);
        if (e == cudaSuccess) {
            uint32_t blocks = std::max(1u, std::min((b->view.pixels + 255) / 256, uint32_t(b->sm_count) * 16));
            k_batch_accumulate<<<blocks, 256, 0, b->stream>>>(b->view, b->counters);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

wf_status capture_batch(wf_batch* b) {
    cudaStream_t st = b->stream;
    uint32_t cap = b->capacity;
    WF_BATCH_CUDA(cudaGraphCreate(&b->graph, 0));
    WF_BATCH_CUDA(cudaStreamBeginCaptureToGraph(st, b->graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    k_batch_raygen<<<std::max(1u, std::min((cap + 255) / 256, uint32_t(b->sm_count) * 16)), 256, 0, st>>>(
        b->view, b->counters, b->paths, b->queue[0], cap);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &captured);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (batch prologue)");
    size_t nodes = 0;
    WF_BATCH_CUDA(cudaGraphGetNodes(b->graph, nullptr, &nodes));
    if (nodes != 1) return fail(WF_ERR_CUDA, "unexpected batch prologue graph (%zu nodes)", nodes);
    cudaGraphNode_t raygen_node = nullptr;
    WF_BATCH_CUDA(cudaGraphGetNodes(b->graph, &raygen_node, &nodes));

    cudaGraphConditionalHandle handle;
    WF_BATCH_CUDA(cudaGraphConditionalHandleCreate(&handle, b->graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop_node = nullptr;
    WF_BATCH_CUDA(cudaGraphAddNode(&loop_node, b->graph, &raygen_node, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];

    WF_BATCH_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    for (uint32_t cur = 0; cur < 2; ++cur) {
        uint32_t nxt = cur ^ 1;
        uint32_t* cur_count = &b->counters->queue_count[cur];
        uint32_t* next_count = &b->counters->queue_count[nxt];
        if (b->opaque)
            k_batch_trace<Opaque<NoTally>><<<batch_grid(b, 0, cap, b->block), b->block, 0, st>>>(
                b->view, b->paths, b->queue[cur], cur_count, b->hit_a, b->hit_inst, b->counters, b->refill);
        else
            k_batch_trace<NoTally><<<batch_grid(b, 0, cap, b->block), b->block, 0, st>>>(
                b->view, b->paths, b->queue[cur], cur_count, b->hit_a, b->hit_inst, b->counters, b->refill);
        if (b->textured)
            k_batch_shade<true><<<batch_grid(b, 1, cap, 128), 128, 0, st>>>(
                b->view, b->paths, b->queue[cur], cur_count, b->hit_a, b->hit_inst, b->terms, b->shade_out,
                b->shadow_origin, b->shadow_dir, b->shadow_capacity, b->counters, next_count);
        else
            k_batch_shade<false><<<batch_grid(b, 1, cap, 128), 128, 0, st>>>(
                b->view, b->paths, b->queue[cur], cur_count, b->hit_a, b->hit_inst, b->terms, b->shade_out,
                b->shadow_origin, b->shadow_dir, b->shadow_capacity, b->counters, next_count);
        if (b->opaque)
            k_batch_shadow<Opaque<NoTally>><<<batch_grid(b, 2, b->shadow_capacity, b->block), b->block, 0, st>>>(
                b->view, b->shadow_origin, b->shadow_dir, b->shadow_result, b->counters, b->shadow_capacity,
                b->refill);
        else
            k_batch_shadow<NoTally><<<batch_grid(b, 2, b->shadow_capacity, b->block), b->block, 0, st>>>(
                b->view, b->shadow_origin, b->shadow_dir, b->shadow_result, b->counters, b->shadow_capacity,
                b->refill);
        k_batch_finalize<<<batch_grid(b, 3, cap, 256), 256, 0, st>>>(
            b->view, b->paths, b->queue[cur], cur_count, b->terms, b->shade_out, b->shadow_result, b->queue[nxt],
            next_count, cap, b->counters);
    }
    unsigned long long bound = (unsigned long long)b->pass_units * b->max_depth / 2 + 2;
    k_batch_condition<<<1, 1, 0, st>>>(handle, b->counters, bound);
    e = cudaStreamEndCapture(st, &captured);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (batch body)");
    WF_BATCH_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return WF_OK;
}

wf_status validate_job(const wf_batch_job& j, uint32_t index) {
    const wf_render_config& c = j.config;
    if (!j.scene) return fail(WF_ERR_INVALID_ARG, "batch job %u: null scene", index);
    if (!std::isfinite(c.indirect_clamp) || c.indirect_clamp < 0.0f)
        return fail(WF_ERR_INVALID_ARG, "batch job %u: indirect radiance clamp must be finite and nonnegative", index);
    if (c.width == 0 || c.height == 0) return fail(WF_ERR_INVALID_ARG, "batch job %u: empty image", index);
    if (c.max_depth == 0 || c.max_depth > kMaxBounces)
        return fail(WF_ERR_INVALID_ARG, "batch job %u: maximum depth must be in [1, %d]", index, kMaxBounces);
    if (c.rng > WF_RNG_PCG32 || c.debug > WF_DEBUG_SHADING_NORMAL)
        return fail(WF_ERR_INVALID_ARG, "batch job %u: unknown rng strategy or debug view", index);
    if (c.caustics) return fail(WF_ERR_UNSUPPORTED, "batch job %u: caustics are not supported in a batch", index);
    if (j.sample_count == 0) return fail(WF_ERR_INVALID_ARG, "batch job %u: empty sample range", index);
    const DeviceScene& v = j.scene->view;
    if (v.punctual_count - v.directional_count > 0 && v.directional_count > 2)
        return fail(WF_ERR_UNSUPPORTED, "batch job %u: more than two directional lights", index);
    return WF_OK;
}

RenderParams job_params(const wf_batch_job& j) {
    const wf_render_config& c = j.config;
    const wf_camera* camera = &j.camera;
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
    return rp;
}

wf_status batch_destroy(wf_batch* b);

wf_status batch_create(const wf_batch_job* jobs, uint32_t count, const wf_batch_config* cfg, void* stream,
                       wf_batch** out) {
    if (!jobs || !out || count == 0) return fail(WF_ERR_INVALID_ARG, "empty batch");
    *out = nullptr;
    wf_batch_config config;
    wf_batch_config_default(&config);
    if (cfg) config = *cfg;
    if (config.block_size > 1024 || (config.block_size && config.block_size % 32))
        return fail(WF_ERR_INVALID_ARG, "batch block size must be a multiple of 32 up to 1024");
    if (config.refill_threshold > 32) return fail(WF_ERR_INVALID_ARG, "refill threshold must be between 0 and 32");
    for (uint32_t i = 0; i < count; ++i)
        if (wf_status e = validate_job(jobs[i], i)) return e;

    // A creation that fails part way frees what it had made.
    std::unique_ptr<wf_batch, wf_status (*)(wf_batch*)> b(new wf_batch(), batch_destroy);
    wf_batch* bp = b.get();
    b->jobs.assign(jobs, jobs + count);
    b->block = config.block_size ? config.block_size : 128u;
    b->refill = config.refill_threshold ? config.refill_threshold : 8u;
    for (uint32_t i = 0; i < count; ++i) {
        b->opaque = b->opaque && !jobs[i].scene->alpha_textures;
        b->textured = b->textured || jobs[i].scene->textured;
    }

    // Unit order: job by job, in the given order or longest per-pixel work first.
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    if (config.longest_first)
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) {
            return uint64_t(jobs[a].sample_count) * jobs[a].config.max_depth >
                   uint64_t(jobs[c].sample_count) * jobs[c].config.max_depth;
        });
    std::vector<BatchJob> host(count);
    uint64_t units = 0, fb = 0, max_directional = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const wf_batch_job& j = jobs[i];
        uint64_t pixels = uint64_t(j.config.width) * j.config.height;
        host[i].scene = j.scene->view;
        host[i].rp = job_params(j);
        host[i].fb_offset = fb;
        host[i].pixels = uint32_t(pixels);
        host[i].sample_start = j.sample_start;
        host[i].sample_count = j.sample_count;
        b->fb_offsets.push_back(fb);
        fb += 3 * pixels;
        b->total_paths += pixels * j.sample_count;
        b->max_depth = std::max(b->max_depth, j.config.max_depth);
        max_directional = std::max<uint64_t>(max_directional, j.scene->view.directional_count);
    }
    // unit order: job by job (in `order`), each job sample by sample
    std::vector<uint32_t> order_arrays(3 * size_t(count));
    uint64_t pixels_total = 0;
    for (uint32_t pos = 0; pos < count; ++pos) {
        uint32_t job = order[pos];
        host[job].unit_begin = uint32_t(units);
        order_arrays[pos] = job;
        order_arrays[count + pos] = uint32_t(units);
        order_arrays[2 * size_t(count) + pos] = uint32_t(pixels_total);
        units += uint64_t(host[job].pixels) * host[job].sample_count;
        pixels_total += host[job].pixels;
        if (units >= 0xffffffffull || pixels_total >= 0xffffffffull)
            return fail(WF_ERR_INVALID_ARG, "batch has 2^32 or more paths");
    }
    b->units = uint32_t(units);
    b->fb_floats = fb;
    b->pass_units = uint32_t(std::min<uint64_t>(units, config.pass_paths ? config.pass_paths : kBatchPassUnits));
    uint64_t cap = config.slot_capacity ? config.slot_capacity : std::min<uint64_t>(units, 4u << 20);
    b->capacity = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(cap, b->pass_units)));

    WF_BATCH_CUDA(cudaGetDevice(&b->device));
    WF_BATCH_CUDA(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device));
    if (stream) {
        b->stream = static_cast<cudaStream_t>(stream);
    } else {
        WF_BATCH_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->own_stream = true;
    }
    uint32_t c = b->capacity;
    WF_BATCH_CUDA(batch_alloc(bp, &b->jobs_dev, count));
    WF_BATCH_CUDA(batch_alloc(bp, &b->order_dev, order_arrays.size()));
    WF_BATCH_CUDA(batch_alloc(bp, &b->view.framebuffer, fb));
    WF_BATCH_CUDA(batch_alloc(bp, &b->view.slot_job, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->view.slot_unit, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->view.unit_radiance, b->pass_units));
    WF_BATCH_CUDA(batch_alloc(bp, &b->paths.origin, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->paths.direction, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->paths.throughput, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->paths.radiance, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->paths.info, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->paths.rng, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->queue[0], c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->queue[1], c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->hit_a, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->hit_inst, c));
    WF_BATCH_CUDA(batch_alloc(bp, &b->terms, size_t(c) * kMaxTerms));
    WF_BATCH_CUDA(batch_alloc(bp, &b->shade_out, c));
    uint64_t shadow = uint64_t(c) * (5u + max_directional);
    b->shadow_capacity = uint32_t(std::min<uint64_t>(shadow, 0xffffffffull));
    WF_BATCH_CUDA(batch_alloc(bp, &b->shadow_origin, b->shadow_capacity));
    WF_BATCH_CUDA(batch_alloc(bp, &b->shadow_dir, b->shadow_capacity));
    WF_BATCH_CUDA(batch_alloc(bp, &b->shadow_result, b->shadow_capacity));
    WF_BATCH_CUDA(batch_alloc(bp, &b->counters, 1));
    WF_BATCH_CUDA(cudaMemcpyAsync(b->jobs_dev, host.data(), sizeof(BatchJob) * count, cudaMemcpyHostToDevice,
                                  b->stream));
    WF_BATCH_CUDA(cudaMemcpyAsync(b->order_dev, order_arrays.data(), sizeof(uint32_t) * order_arrays.size(),
                                  cudaMemcpyHostToDevice, b->stream));
    WF_BATCH_CUDA(cudaMemsetAsync(b->view.framebuffer, 0, sizeof(float) * fb, b->stream));
    WF_BATCH_CUDA(cudaMemsetAsync(b->counters, 0, sizeof(Counters), b->stream));
    b->paths.slot_sample = nullptr;
    b->paths.wait = nullptr;
    b->view.jobs = b->jobs_dev;
    b->view.job_order = b->order_dev;
    b->view.order_units = b->order_dev + count;
    b->view.order_pixels = b->order_dev + 2 * size_t(count);
    b->view.job_count = count;
    b->view.units = b->units;
    b->view.pixels = uint32_t(pixels_total);
    WF_BATCH_CUDA(b->opaque ? batch_resident(bp, 0, k_batch_trace<Opaque<NoTally>>, b->block)
                            : batch_resident(bp, 0, k_batch_trace<NoTally>, b->block));
    WF_BATCH_CUDA(b->textured ? batch_resident(bp, 1, k_batch_shade<true>, 128)
                              : batch_resident(bp, 1, k_batch_shade<false>, 128));
    WF_BATCH_CUDA(b->opaque ? batch_resident(bp, 2, k_batch_shadow<Opaque<NoTally>>, b->block)
                            : batch_resident(bp, 2, k_batch_shadow<NoTally>, b->block));
    WF_BATCH_CUDA(batch_resident(bp, 3, k_batch_finalize, 256));
    if (wf_status e = capture_batch(bp)) {
        abandon_capture(b->stream);
        return e;
    }
    WF_BATCH_CUDA(cudaStreamSynchronize(b->stream));
    *out = b.release();
    return WF_OK;
}

wf_status batch_destroy(wf_batch* b) {
    if (!b) return WF_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void* p : b->allocations) cudaFree(p);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return WF_OK;
}

}  // namespace
}  // namespace wf

using namespace wf;

extern "C" void wf_batch_config_default(wf_batch_config* config) {
    if (!config) return;
    std::memset(config, 0, sizeof(*config));
    config->longest_first = 1;
}

extern "C" wf_status wf_batch_create(const wf_batch_job* jobs, uint32_t job_count, const wf_batch_config* config,
                                     void* stream, wf_batch** out) {
    wf_batch* b = nullptr;
    wf_status e = batch_create(jobs, job_count, config, stream, &b);
    if (e != WF_OK) return e;
    *out = b;
    return WF_OK;
}

extern "C" wf_status wf_batch_run(wf_batch* b) {
    if (!b) return fail(WF_ERR_INVALID_ARG, "null batch");
    WF_BATCH_CUDA(batch_run(b));
    return WF_OK;
}

extern "C" wf_status wf_batch_synchronize(wf_batch* b) {
    if (!b) return fail(WF_ERR_INVALID_ARG, "null batch");
    WF_BATCH_CUDA(cudaStreamSynchronize(b->stream));
    uint32_t flags[2] = {0, 0};
    WF_BATCH_CUDA(cudaMemcpyAsync(&flags[0], &b->counters->overflow, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  b->stream));
    WF_BATCH_CUDA(cudaMemcpyAsync(&flags[1], &b->counters->error, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  b->stream));
    WF_BATCH_CUDA(cudaStreamSynchronize(b->stream));
    if (flags[1]) return fail(WF_ERR_TIMEOUT, "batch loop exceeded its iteration bound");
    if (flags[0]) return fail(WF_ERR_CAPACITY, "shadow queue or term buffer overflow (flags %u)", flags[0]);
    return WF_OK;
}

extern "C" wf_status wf_batch_reset(wf_batch* b) {
    if (!b) return fail(WF_ERR_INVALID_ARG, "null batch");
    WF_BATCH_CUDA(cudaMemsetAsync(b->view.framebuffer, 0, sizeof(float) * b->fb_floats, b->stream));
    return WF_OK;
}

extern "C" wf_status wf_batch_download(wf_batch* b, uint32_t job, float* rgb) {
    if (!b || !rgb) return fail(WF_ERR_INVALID_ARG, "null argument");
    if (job >= b->jobs.size()) return fail(WF_ERR_INVALID_ARG, "batch job %u out of range", job);
    const wf_render_config& c = b->jobs[job].config;
    WF_BATCH_CUDA(cudaMemcpyAsync(rgb, b->view.framebuffer + b->fb_offsets[job],
                                  sizeof(float) * 3 * size_t(c.width) * c.height, cudaMemcpyDeviceToHost, b->stream));
    return wf_batch_synchronize(b);
}

extern "C" wf_status wf_batch_framebuffer_device(wf_batch* b, uint32_t job, float** rgb) {
    if (!b || !rgb) return fail(WF_ERR_INVALID_ARG, "null argument");
    if (job >= b->jobs.size()) return fail(WF_ERR_INVALID_ARG, "batch job %u out of range", job);
    *rgb = b->view.framebuffer + b->fb_offsets[job];
    return WF_OK;
}

extern "C" wf_status wf_batch_stats(wf_batch* b, wf_render_stats* stats, uint32_t reset) {
    if (!b || !stats) return fail(WF_ERR_INVALID_ARG, "null argument");
    unsigned long long v[4];
    WF_BATCH_CUDA(cudaMemcpyAsync(v, &b->counters->extension_rays, sizeof(v), cudaMemcpyDeviceToHost, b->stream));
    WF_BATCH_CUDA(cudaStreamSynchronize(b->stream));
    stats->extension_rays = v[0];
    stats->shadow_rays = v[1];
    stats->paths = v[2];
    stats->kernel_launches = v[3];
    if (reset) {
        WF_BATCH_CUDA(cudaMemsetAsync(&b->counters->extension_rays, 0, sizeof(v), b->stream));
        WF_BATCH_CUDA(cudaStreamSynchronize(b->stream));
    }
    return WF_OK;
}

extern "C" wf_status wf_batch_destroy(wf_batch* b) { return batch_destroy(b); }

extern "C" wf_status wf_batch_autotune(const wf_batch_job* jobs, uint32_t job_count, const uint32_t* slot_capacities,
                                       const uint32_t* block_sizes, const uint32_t* refill_thresholds, void* stream,
                                       wf_batch_config* best, float* times_ms, uint32_t times_capacity) {
    if (!best) return fail(WF_ERR_INVALID_ARG, "null result");
    static const uint32_t kCaps[] = {0, 0};
    static const uint32_t kBlocks[] = {128, 0};
    static const uint32_t kRefills[] = {8, 0};
    const uint32_t* caps = slot_capacities ? slot_capacities : kCaps;
    const uint32_t* blocks = block_sizes ? block_sizes : kBlocks;
    const uint32_t* refills = refill_thresholds ? refill_thresholds : kRefills;
    auto list = [](const uint32_t* l, bool zero_ok) {
        std::vector<uint32_t> v;
        if (zero_ok && l[0] == 0) return std::vector<uint32_t>{0u};
        for (; *l; ++l) v.push_back(*l);
        return v;
    };
    std::vector<uint32_t> cap_list = list(caps, true), block_list = list(blocks, false),
                          refill_list = list(refills, false);
    if (block_list.empty() || refill_list.empty()) return fail(WF_ERR_INVALID_ARG, "empty candidate list");
    float best_ms = 0.0f;
    uint32_t index = 0;
    bool have = false;
    for (uint32_t cap : cap_list)
        for (uint32_t block : block_list)
            for (uint32_t refill_at : refill_list) {
                wf_batch_config cfg;
                wf_batch_config_default(&cfg);
                cfg.slot_capacity = cap;
                cfg.block_size = block;
                cfg.refill_threshold = refill_at;
                wf_batch* b = nullptr;
                if (wf_status e = batch_create(jobs, job_count, &cfg, stream, &b)) return e;
                cudaEvent_t e0 = nullptr, e1 = nullptr;
                float ms = 0.0f;
                cudaError_t err = cudaEventCreate(&e0);
                if (err == cudaSuccess) err = cudaEventCreate(&e1);
                if (err == cudaSuccess) err = cudaEventRecord(e0, b->stream);
                if (err == cudaSuccess) err = batch_run(b);
                if (err == cudaSuccess) err = cudaEventRecord(e1, b->stream);
                if (err == cudaSuccess) err = cudaEventSynchronize(e1);
                if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
                if (e0) cudaEventDestroy(e0);
                if (e1) cudaEventDestroy(e1);
                wf_status sync = err == cudaSuccess ? wf_batch_synchronize(b) : cuda_fail(err, "autotune run");
                batch_destroy(b);
                if (sync != WF_OK) return sync;
                if (times_ms && index < times_capacity) times_ms[index] = ms;
                ++index;
                if (!have || ms < best_ms) {
                    have = true;
                    best_ms = ms;
                    *best = cfg;
                }
            }
    return WF_OK;
}
