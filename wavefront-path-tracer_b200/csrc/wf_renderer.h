// Renderer object behind the C ABI (host side).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "wf_internal.h"

namespace wf {

struct TileDev {
    uint32_t x, y, width, height;
    uint32_t advance_sample;  // add `samples` to the sample index after the launch
    uint32_t samples = 1;     // streaming mode: samples per pixel of this launch
};

// Device counters of one renderer (one allocation, zeroed at creation).
constexpr int kMaxBounces = 64;
constexpr uint32_t kDefaultRegeneratePercent = 25;  // streaming mode (wf_render_config::regenerate_percent)
constexpr uint32_t kErrorBarrierTimeout = 1;  // a persistent-kernel grid barrier wait gave up
constexpr uint32_t kErrorStreamBound = 2;     // the streaming loop exceeded samples * max_depth bounces
struct Counters {
    uint32_t queue_count[2];
    uint32_t shadow_count;
    uint32_t overflow;
    uint32_t sample_index;
    uint32_t error;          // kErrorBarrierTimeout / kErrorStreamBound
    uint32_t barrier_count;
    uint32_t barrier_generation;
    uint32_t work_trace;   // dynamic work counters (32-entry chunks per warp)
    uint32_t work_shade;
    uint32_t work_shadow;
    uint32_t stream_iterations;  // streaming mode: loop iterations of the current launch
    uint32_t gather_count;       // caustic gather requests of the current bounce
    uint32_t work_gather;
    uint32_t dense_count;        // gather requests deferred to the warp-per-request kernel
    uint32_t work_dense;
    uint32_t shade_bucket[8];    // queue entries per shading category (current bounce)
    uint32_t shade_cursor[8];
    uint32_t next_unit;          // job batch: next (job, sample, pixel) unit to start
    uint32_t pass_begin, pass_end;  // job batch: the units of the current pass
    unsigned long long extension_rays;
    unsigned long long shadow_rays;
    unsigned long long paths;
    unsigned long long kernel_launches;  // launches of the render kernels (each CTA 0 thread 0 adds one)
    uint32_t profile[kMaxBounces];          // per-bounce queue sizes (latest sample)
    uint32_t persistent_count[kMaxBounces + 1];
    uint32_t persistent_work[kMaxBounces + 1];
    // Streaming mode: camera rays of slots that started a new sample, queued
    // after queue_count[q] survivors of queue q (merged into the queue once
    // traced), and the work counter of the per-thread camera-ray trace.
    uint32_t camera_count[2];
    uint32_t work_camera;
    // Bounds of the device-side waits (wf_renderer_set_watchdog); 0 = default.
    unsigned long long barrier_limit;  // cycles a grid-barrier wait may take (default 2^31)
    uint32_t stream_limit;             // streaming-loop passes per launch (default: samples x depth bound)
};

// Traversal work totals of one profiling pass: node visits, triangle tests,
// sphere tests, instance entries.
struct TallyTotals {
    unsigned long long v[4];
};

struct PathSoA {
    float4* origin;     // xyz, prev_pdf
    float4* direction;  // xyz, eta_scale
    float4* throughput; // xyz, medium_density
    float4* radiance;   // xyz, -
    uint4* info;        // pixel, depth, medium, flags (1 = specular, 2 = active)
    unsigned long long* rng;
    uint32_t* slot_sample;  // streaming mode: sample of the slot's path, relative to the launch's first
    uint8_t* wait;          // streaming mode: 1 = the slot's path ended and its next sample has not started
};

struct AsyncCheckpointSlot {
    float* pixels = nullptr;
    cudaEvent_t copied = nullptr;
    std::atomic<bool> busy{false};
    std::thread writer;
};

}  // namespace wf

struct wf_renderer {
    const wf_scene* scene = nullptr;
    wf_render_config config{};
    wf::RenderParams params{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool opaque = true;     // no alpha-textured material: the Opaque<> trace and shadow kernels
    bool textured = false;  // some textured material: k_shade<true>
    bool sort_shading = true;  // material-sort the hits before shading (k_classify, k_scatter)
    int device = 0;
    int sm_count = 148;
    uint32_t capacity = 0;       // path slots: tile_capacity x wave
    uint32_t tile_capacity = 0;  // pixels of the largest tile
    uint32_t wave = 1;           // graph mode: samples per launch of the bounce chain (samples_per_wave)
    uint32_t block_trace = 128, block_shade = 128, block_finalize = 256, block_gather = 128, block_camera = 128;
    uint32_t grid_cap = 0;
    std::vector<void*> allocations;
    uint64_t device_bytes = 0;
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
    wf::TileDev* tile = nullptr;
    float* framebuffer = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    // capture-time fork of the caustic gathers beside the shadow rays
    cudaStream_t side = nullptr;
    cudaEvent_t fork_event = nullptr, join_event = nullptr;
    uint32_t grid_resident[6] = {0, 0, 0, 0, 0, 0};  // trace, shade, shadow, finalize, gather, camera-ray trace
    uint8_t* shade_key = nullptr;     // shading category of each queue entry
    uint32_t* shade_order = nullptr;  // queue entries grouped by category (the order k_shade takes them)
    wf::GatherQueue gathers{};                      // caustic gather requests (graph and streaming modes)
    uint32_t persistent_blocks = 0;  // resident grid of the fused persistent kernel
    uint32_t phased_blocks = 0;      // resident grid of the staged persistent kernel
    uint32_t persistent_block_size = 128;
    uint32_t chunk = 1;
    uint32_t refill = 8;  // trace/shadow kernels: idle lanes of a warp that trigger a refill
    uint32_t regenerate_percent = 25;  // streaming mode: see wf_render_config::regenerate_percent
    // photon map
    uint32_t photons_emitted = 0, photons_stored = 0;
    float4* photon_raw = nullptr;  // 4 float4 per photon: pos(.w valid), dir, flux, rng/meta
    // checkpoint writer
    std::vector<std::unique_ptr<wf::AsyncCheckpointSlot>> slots;
    std::mutex write_mutex;
    uint32_t latest_written = 0;
    uint32_t last_tile_width = 0, last_tile_height = 0;
    wf::TallyTotals* tally = nullptr;  // [0] closest hit, [1] any hit (profiling pass)
    // Graph mode with two wavefronts: the twin has its own buffers, graph and
    // stream, renders into this renderer's framebuffer and reuses its photon
    // map; each render call splits its rows between the two.
    wf_renderer* twin = nullptr;
    bool external_framebuffer = false;
    uint32_t last_tile_parts = 1;  // which of {this, twin} rendered the last tile (bit 0, bit 1)
    cudaEvent_t twin_fork = nullptr, twin_join = nullptr;
    // wf_framebuffer_download_async: two device snapshots of the framebuffer
    // and the stream that copies them to the host
    float* snapshot[2] = {nullptr, nullptr};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snapshot_ready[2] = {nullptr, nullptr}, copy_done[2] = {nullptr, nullptr};
    uint32_t next_snapshot = 0;
};

namespace wf {
// After a failed graph capture: ends the capture if it is still open
// (discarding its graph) and consumes the launch error it recorded, so
// neither outlives the failed call on the calling thread.
inline void abandon_capture(cudaStream_t st) {
    cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &status) == cudaSuccess && status != cudaStreamCaptureStatusNone) {
        cudaGraph_t partial = nullptr;
        cudaStreamEndCapture(st, &partial);
        if (partial) cudaGraphDestroy(partial);
    }
    cudaGetLastError();
}

wf_status renderer_create(const wf_scene* scene, const wf_camera* camera, const wf_render_config* config,
                          void* stream, wf_renderer** out);
wf_status renderer_destroy(wf_renderer* r);
wf_status renderer_render(wf_renderer* r, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_start,
                          uint32_t sample_count, uint32_t clear);
wf_status renderer_render_frame(wf_renderer* r, uint32_t sample_count);
wf_status renderer_profile(wf_renderer* r, wf_kernel_profile* out);
// The renderers that hold device counters: the renderer and its twin.
inline int renderer_parts(wf_renderer* r, wf_renderer* parts[2]) {
    parts[0] = r;
    parts[1] = r->twin;
    return r->twin ? 2 : 1;
}
wf_status trace_closest_batch(const wf_scene* scene, const wf_ray* rays, uint32_t count, wf_hit* hits,
                              cudaStream_t stream);
wf_status trace_any_batch(const wf_scene* scene, const wf_ray* rays, const float* max_distance, uint32_t count,
                          uint8_t* occluded, cudaStream_t stream);
wf_status cuda_fail(cudaError_t e, const char* what);
wf_status frame_guides(const wf_scene* scene, const wf_camera* camera, const wf_camera* previous, uint32_t width,
                       uint32_t height, uint32_t x, uint32_t y, uint32_t w, uint32_t h, wf_frame_guide* guides,
                       cudaStream_t stream);
}  // namespace wf
