// Path-state access and work distribution shared by the wavefront kernels
// (single-scene renderer and the job batch).
#pragma once

#include "wf_renderer.h"
#include "wf_shade.cuh"

namespace wf {

// Device-side launch count of the render kernels (thread 0 of CTA 0 adds
// one; graph branches can run two kernels at once).
WF_DEV void count_launch(Counters* c) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&c->kernel_launches, 1ull);
}

WF_DEV Path load_path(const PathSoA& ps, uint32_t p) {
    float4 o = ps.origin[p], d = ps.direction[p], t = ps.throughput[p];
    uint4 info = ps.info[p];
    Path path;
    path.origin = f4xyz(o);
    path.prev_pdf = o.w;
    path.direction = f4xyz(d);
    path.eta_scale = d.w;
    path.throughput = f4xyz(t);
    path.medium_density = t.w;
    path.pixel = info.x;
    path.depth = info.y;
    path.medium = info.z;
    path.specular = (info.w & 1u) != 0;
    path.active = (info.w & 2u) != 0;
    path.rng = ps.rng[p];
    return path;
}

WF_DEV void store_path(const PathSoA& ps, uint32_t p, const Path& path) {
    ps.origin[p] = make_float4(path.origin.x, path.origin.y, path.origin.z, path.prev_pdf);
    ps.direction[p] = make_float4(path.direction.x, path.direction.y, path.direction.z, path.eta_scale);
    ps.throughput[p] = make_float4(path.throughput.x, path.throughput.y, path.throughput.z, path.medium_density);
    ps.info[p] = make_uint4(path.pixel, path.depth, path.medium, (path.specular ? 1u : 0u) | (path.active ? 2u : 0u));
    ps.rng[p] = path.rng;
}

// generatePrimaryRays, src/renderer/renderer.cu:10-42.
WF_DEV void init_path(const RenderParams& rp, const TileDev& tile, uint32_t sample, uint32_t lp, Path& path) {
    uint32_t x = tile.x + lp % tile.width;
    uint32_t y = tile.y + lp / tile.width;
    uint32_t pixel = y * rp.width + x;
    uint64_t rng = make_rng_state(pixel_rng_key(pixel, sample, rp.rng), rp.rng);
    float u = (float(x) + random_float(rng, rp.rng)) / float(rp.width);
    float v = (float(y) + random_float(rng, rp.rng)) / float(rp.height);
    camera_ray(rp.camera, u, v, path.origin, path.direction);
    path.throughput = V3{1.0f, 1.0f, 1.0f};
    path.pixel = pixel;
    path.depth = 0;
    path.rng = rng;
    path.medium = kInvalid;
    path.medium_density = 1.0f;
    path.prev_pdf = 0.0f;
    path.specular = true;
    path.active = true;
    path.eta_scale = 1.0f;
}

// Warps pull 32-entry chunks from `counter` until `n` is exhausted (the
// counter is zeroed by the kernel that runs before).  Balances warps whose
// rays need very different traversal work.
WF_DEV bool next_chunk(uint32_t* counter, uint32_t n, uint32_t& base) {
    uint32_t b = 0;
    if ((threadIdx.x & 31) == 0) b = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, b, 0);
    return base < n;
}

// Sums a thread's tally into per-launch totals (profiling pass only).
WF_DEV void flush_tally(const CountTally& t, TallyTotals* totals) {
    unsigned long long v[4] = {t.nodes, t.triangles, t.spheres, t.instances};
    for (int k = 0; k < 4; ++k) {
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
        if ((threadIdx.x & 31) == 0 && v[k]) atomicAdd(&totals->v[k], v[k]);
    }
}

}  // namespace wf
