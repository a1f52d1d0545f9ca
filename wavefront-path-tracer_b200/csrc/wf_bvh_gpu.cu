// GPU BVH2 builder: PLOC (Meister and Bittner, "Parallel Locally-Ordered
// Clustering for Bounding Volume Hierarchy Construction", IEEE TVCG 2018).
//
// The reference builds its BVH2s on the GPU with NexusBVH (an H-PLOC builder
// in an un-vendored submodule, called at src/scene/scene.cu:148-149,227-228,
// 262-264).  This is this build's GPU builder for the same role:
//   1. primitive centroids are quantised to 21 bits per axis (one scale,
//      the widest extent, for all axes) and interleaved into 63-bit Morton
//      keys;
//   2. a stable LSD radix sort (8-bit digits, hand-written) orders the
//      primitives along the curve;
//   3. clusters start as one leaf per primitive in that order; each round,
//      every cluster finds the neighbour within +-kPlocRadius positions whose
//      union box has the smallest surface area (symmetric tie-breaks, see
//      k_nearest), mutual nearest neighbours merge into a new node (the
//      lower position keeps it), and an exclusive scan compacts the
//      survivors and numbers the new nodes;
//   4. rounds repeat until one cluster is left (at most kMaxRounds; the
//      caller falls back to the host builder beyond that);
//   5. treelet restructuring (k_restructure) lowers the tree's SAH cost,
//      and the leaf depth is measured on the device before the download;
//   6. the host's binned-SAH builder rebuilds the levels above the largest
//      subtrees of at most kTopClusterLeaves leaves (rebuild_top).
// Every step is deterministic (stable sort, index tie-breaks, scan-ordered
// node numbering, subtree-local treelet choices), so a scene always gets the
// same tree.  The output is the host builder's format (bvh_build.h): 2n-1
// nodes, leaves first with left == kInvalidChild and right == primitive, the
// root last (after restructuring, a child may follow its parent).
#include "bvh_build.h"
#include "wf_bvh_gpu.h"
#include "wf_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace wf {
namespace {

constexpr int kPlocRadius = 16;
constexpr int kSortThreads = 256;
constexpr int kSortChunks = 16;  // elements per sort block = threads x chunks
constexpr int kSortTile = kSortThreads * kSortChunks;
constexpr int kScanThreads = 1024;
constexpr int kNearestThreads = 256;
constexpr int kMaxRounds = 512;

__device__ __forceinline__ float half_area(const BvhBox& b) {
    float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ BvhBox merged(const BvhBox& a, const BvhBox& b) {
    BvhBox r;
    for (int k = 0; k < 3; ++k) {
        r.lo[k] = fminf(a.lo[k], b.lo[k]);
        r.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    return r;
}

// Floats as order-preserving unsigned integers, for atomicMin/atomicMax.
__device__ __forceinline__ uint32_t ordered(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ inline float unordered(uint32_t u) {
    uint32_t v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    memcpy(&f, &v, 4);
    return f;
}

// Centroid bounds: bounds[0..2] = ordered min, bounds[3..5] = ordered max.
__global__ void k_centroid_bounds(const BvhBox* prims, uint32_t n, uint32_t* bounds) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int k = 0; k < 3; ++k) {
            float c = 0.5f * (prims[i].lo[k] + prims[i].hi[k]);
            lo[k] = fminf(lo[k], c);
            hi[k] = fmaxf(hi[k], c);
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], off));
            hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(&bounds[k], ordered(lo[k]));
            atomicMax(&bounds[3 + k], ordered(hi[k]));
        }
    }
}

__device__ __forceinline__ unsigned long long spread21(uint32_t v) {
    unsigned long long x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void k_morton(const BvhBox* prims, uint32_t n, const uint32_t* bounds, unsigned long long* keys,
                         uint32_t* values) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // One scale for all three axes (the widest extent), so that the curve
    // follows physical distance: per-axis scales would give a flat scene's
    // thin axis (a heightfield's height) as many bits as its wide ones and
    // scatter neighbours along the curve.
    uint32_t q[3];
    float extent = 0.0f;
    for (int k = 0; k < 3; ++k) extent = fmaxf(extent, unordered(bounds[3 + k]) - unordered(bounds[k]));
    for (int k = 0; k < 3; ++k) {
        float lo = unordered(bounds[k]);
        float c = 0.5f * (prims[i].lo[k] + prims[i].hi[k]);
        float t = extent > 0.0f ? (c - lo) / extent : 0.0f;
        t = fminf(fmaxf(t, 0.0f), 1.0f);
        q[k] = min(uint32_t(t * 2097151.0f), 2097151u);
    }
    keys[i] = spread21(q[0]) | spread21(q[1]) << 1 | spread21(q[2]) << 2;
    values[i] = i;
}

// ---------------------------------------------------------- radix sort
// Per-block digit histograms, digit-major: hist[digit * blocks + block].
__global__ void k_sort_histogram(const unsigned long long* keys, uint32_t n, int shift, uint32_t* hist) {
    __shared__ uint32_t count[256];
    for (int d = threadIdx.x; d < 256; d += blockDim.x) count[d] = 0;
    __syncthreads();
    uint32_t base = blockIdx.x * kSortTile;
    for (int c = 0; c < kSortChunks; ++c) {
        uint32_t i = base + c * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&count[(keys[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[size_t(d) * gridDim.x + blockIdx.x] = count[d];
}

// Stable scatter: within a tile, elements keep their order per digit (warp
// match ranks, then warps in order, then chunks in order).
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const unsigned long long* keys_in,
                                                               const uint32_t* values_in, uint32_t n, int shift,
                                                               const uint32_t* offsets,
                                                               unsigned long long* keys_out,
                                                               uint32_t* values_out) {
    constexpr int kWarps = kSortThreads / 32;
    __shared__ uint32_t running[256];
    __shared__ uint32_t warp_count[kWarps][256];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = threadIdx.x; d < 256; d += blockDim.x) running[d] = offsets[size_t(d) * gridDim.x + blockIdx.x];
    for (int k = threadIdx.x; k < kWarps * 256; k += blockDim.x) (&warp_count[0][0])[k] = 0;
    __syncthreads();
    uint32_t base = blockIdx.x * kSortTile;
    for (int c = 0; c < kSortChunks; ++c) {
        uint32_t i = base + c * kSortThreads + threadIdx.x;
        bool valid = i < n;
        unsigned long long key = valid ? keys_in[i] : 0ull;
        uint32_t value = valid ? values_in[i] : 0u;
        uint32_t digit = valid ? uint32_t((key >> shift) & 0xffu) : 256u;
        unsigned peers = __match_any_sync(0xffffffffu, digit);
        uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && lane == __ffs(peers) - 1) warp_count[warp][digit] = __popc(peers);
        __syncthreads();
        for (int d = threadIdx.x; d < 256; d += blockDim.x) {
            uint32_t run = running[d];
            for (int w = 0; w < kWarps; ++w) {
                uint32_t t = warp_count[w][d];
                warp_count[w][d] = run;
                run += t;
            }
            running[d] = run;
        }
        __syncthreads();
        if (valid) {
            uint32_t pos = warp_count[warp][digit] + rank;
            keys_out[pos] = key;
            values_out[pos] = value;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kWarps * 256; k += blockDim.x) (&warp_count[0][0])[k] = 0;
        __syncthreads();
    }
}

// ------------------------------------------------------------------ scan
// Exclusive scan of one kScanThreads-element block; block sums to `sums`.
__global__ void __launch_bounds__(kScanThreads) k_scan_block(const uint32_t* in, uint32_t* out, uint32_t n,
                                                             uint32_t* sums) {
    __shared__ uint32_t warp_sum[kScanThreads / 32];
    uint32_t i = blockIdx.x * kScanThreads + threadIdx.x;
    uint32_t v = i < n ? in[i] : 0u;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = warp_sum[lane];
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, off);
            if (lane >= off) s += y;
        }
        warp_sum[lane] = s;
    }
    __syncthreads();
    uint32_t warp_base = warp ? warp_sum[warp - 1] : 0u;
    if (i < n) out[i] = warp_base + x - v;
    if (threadIdx.x == kScanThreads - 1 && sums) sums[blockIdx.x] = warp_base + x;
}

__global__ void k_scan_add(uint32_t* data, uint32_t n, const uint32_t* block_offsets) {
    uint32_t i = blockIdx.x * kScanThreads + threadIdx.x;
    if (i < n && blockIdx.x > 0) data[i] += block_offsets[blockIdx.x];
}

struct Scratch {
    std::vector<void*> blocks;
    cudaError_t error = cudaSuccess;
    template <typename T>
    T* alloc(size_t count) {
        void* p = nullptr;
        if (error == cudaSuccess) error = device_alloc(&p, sizeof(T) * std::max<size_t>(count, 1));
        if (error == cudaSuccess) blocks.push_back(p);
        return static_cast<T*>(p);
    }
    ~Scratch() {
        for (void* p : blocks) cudaFree(p);
    }
};

// Exclusive scan of n values in place-free form (in -> out), any n.
cudaError_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t st, Scratch& scratch) {
    if (n == 0) return cudaSuccess;
    uint32_t blocks = (n + kScanThreads - 1) / kScanThreads;
    uint32_t* sums = blocks > 1 ? scratch.alloc<uint32_t>(blocks) : nullptr;
    if (scratch.error != cudaSuccess) return scratch.error;
    k_scan_block<<<blocks, kScanThreads, 0, st>>>(in, out, n, sums);
    if (blocks == 1) return cudaGetLastError();
    uint32_t* sum_offsets = scratch.alloc<uint32_t>(blocks);
    if (scratch.error != cudaSuccess) return scratch.error;
    if (cudaError_t e = exclusive_scan(sums, sum_offsets, blocks, st, scratch)) return e;
    k_scan_add<<<blocks, kScanThreads, 0, st>>>(out, n, sum_offsets);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ PLOC
__global__ void k_leaves(const BvhBox* prims, const uint32_t* order, uint32_t n, BvhBinaryNode* nodes,
                         uint32_t* clusters, BvhBox* boxes) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    nodes[i] = BvhBinaryNode{prims[i], kInvalidChild, i};
    uint32_t p = order[i];
    clusters[i] = p;
    boxes[i] = prims[p];
}

// Nearest neighbour of every cluster within +-kPlocRadius: the candidate
// with the smallest key (union surface area, distance in the curve order,
// not being the position's pair partner i^1, lower position).  The key is
// symmetric in the two positions, so the pair with the smallest key over the
// whole array is mutual and every round merges at least once; clusters with
// equal boxes pair up as (2k, 2k+1) and halve each round.  Boxes of the
// block's clusters and the halo are staged in shared memory.
__global__ void __launch_bounds__(kNearestThreads) k_nearest(const BvhBox* boxes, uint32_t m, uint32_t* nearest) {
    __shared__ BvhBox tile[kNearestThreads + 2 * kPlocRadius];
    int first = int(blockIdx.x * kNearestThreads) - kPlocRadius;
    for (int k = threadIdx.x; k < kNearestThreads + 2 * kPlocRadius; k += blockDim.x) {
        int j = first + k;
        if (j >= 0 && j < int(m)) tile[k] = boxes[j];
    }
    __syncthreads();
    int i = int(blockIdx.x * kNearestThreads + threadIdx.x);
    if (i >= int(m)) return;
    const BvhBox& mine = tile[threadIdx.x + kPlocRadius];
    float best = INFINITY;
    int best_j = -1, best_d = 0, best_other = 0;
    int lo = max(0, i - kPlocRadius), hi = min(int(m) - 1, i + kPlocRadius);
    for (int j = lo; j <= hi; ++j) {  // ascending j: equal keys keep the lower position
        if (j == i) continue;
        float a = half_area(merged(mine, tile[j - first]));
        int d = abs(j - i), other = j != (i ^ 1);
        bool better = best_j < 0 || a < best || (a == best && (d < best_d || (d == best_d && other < best_other)));
        if (better) {
            best = a;
            best_j = j;
            best_d = d;
            best_other = other;
        }
    }
    nearest[i] = uint32_t(best_j < 0 ? i : best_j);
}

// alive: not the upper half of a mutual pair; leader: lower half of one.
__global__ void k_merge_flags(const uint32_t* nearest, uint32_t m, uint32_t* alive, uint32_t* leader) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t j = nearest[i];
    bool mutual = j != i && nearest[j] == i;
    alive[i] = mutual && i > j ? 0u : 1u;
    leader[i] = mutual && i < j ? 1u : 0u;
}

// Survivors move to their compacted position; each mutual pair becomes a new
// node.
__global__ void k_merge(const uint32_t* clusters, const BvhBox* boxes, const uint32_t* nearest, uint32_t m,
                        const uint32_t* alive, const uint32_t* alive_at, const uint32_t* leader,
                        const uint32_t* leader_at, uint32_t node_base, BvhBinaryNode* nodes, uint32_t* clusters_out,
                        BvhBox* boxes_out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !alive[i]) return;
    uint32_t dst = alive_at[i];
    if (leader[i]) {
        uint32_t j = nearest[i];
        BvhBox box = merged(boxes[i], boxes[j]);
        uint32_t node = node_base + leader_at[i];
        nodes[node] = BvhBinaryNode{box, clusters[i], clusters[j]};
        clusters_out[dst] = node;
        boxes_out[dst] = box;
    } else {
        clusters_out[dst] = clusters[i];
        boxes_out[dst] = boxes[i];
    }
}

// ------------------------------------------------- treelet restructuring
// Karras and Aila, "Fast Parallel Construction of High-Quality Bounding
// Volume Hierarchies" (HPG 2013): after PLOC, one thread per leaf walks up
// the tree; the second thread to reach a node owns it (both subtrees are
// final by then).  A node with at least `min_leaves` leaves below it roots
// a treelet: starting from its two children, the treelet leaf with the
// largest surface area is expanded until there are kTreeletLeaves of them.
// A dynamic programme over the 2^7 subsets of those leaves finds the
// topology with the smallest summed surface area of its internal nodes
// (the SAH with unit costs; the leaves' subtrees are fixed), and the
// treelet's internal node slots are rewired to it if it beats the current
// one.  A treelet only touches nodes below its root, which no other thread
// reads or writes any more, and every choice is a pure function of that
// subtree (ties keep the first split found), so the result does not depend
// on thread timing.  Loads bypass L1 (__ldcg): another SM wrote the data.
constexpr int kTreeletLeaves = 7;
constexpr int kTreeletSubsets = 1 << kTreeletLeaves;
constexpr int kRestructureRounds = 3;  // treelet roots with >= 7, 14, 28 leaves
constexpr int kRestructureThreads = 128;

__device__ __forceinline__ BvhBinaryNode load_node(const BvhBinaryNode* nodes, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    float4 a = __ldcg(p), b = __ldcg(p + 1);
    BvhBinaryNode n;
    n.box.lo[0] = a.x;
    n.box.lo[1] = a.y;
    n.box.lo[2] = a.z;
    n.box.hi[0] = a.w;
    n.box.hi[1] = b.x;
    n.box.hi[2] = b.y;
    n.left = __float_as_uint(b.z);
    n.right = __float_as_uint(b.w);
    return n;
}

__device__ __forceinline__ void store_node(BvhBinaryNode* nodes, uint32_t i, const BvhBox& box, uint32_t left,
                                           uint32_t right) {
    float4* p = reinterpret_cast<float4*>(nodes + i);
    __stcg(p, make_float4(box.lo[0], box.lo[1], box.lo[2], box.hi[0]));
    __stcg(p + 1, make_float4(box.hi[1], box.hi[2], __uint_as_float(left), __uint_as_float(right)));
}

// parent[] of every node (the root's stays kInvalidChild, set by the caller).
__global__ void k_parents(const BvhBinaryNode* nodes, uint32_t n, uint32_t* parent) {
    uint32_t i = n + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n - 1) return;
    parent[nodes[i].left] = i;
    parent[nodes[i].right] = i;
}

// Leaves: subtree cost = own half area, one leaf.
__global__ void k_leaf_costs(const BvhBinaryNode* nodes, uint32_t n, float* cost, uint32_t* leafcount) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cost[i] = half_area(nodes[i].box);
    leafcount[i] = 1;
}

// Restructures the treelet rooted at internal node `root`; returns the
// subtree's cost (summed half areas of its nodes).
__device__ float optimize_treelet(BvhBinaryNode* nodes, uint32_t* parent, float* cost, uint32_t* leafcount,
                                  uint32_t root, const BvhBinaryNode& top) {
    uint32_t leaf[kTreeletLeaves], inner[kTreeletLeaves - 1], count[kTreeletLeaves];
    BvhBox box[kTreeletLeaves];
    float sub[kTreeletLeaves];
    bool expandable[kTreeletLeaves];
    int nl = 0, ni = 1;
    inner[0] = root;
    float old_cost = half_area(top.box);
    auto add = [&](int slot, uint32_t node) {
        BvhBinaryNode x = load_node(nodes, node);
        leaf[slot] = node;
        box[slot] = x.box;
        expandable[slot] = x.left != kInvalidChild;
        sub[slot] = __ldcg(cost + node);
        count[slot] = __ldcg(leafcount + node);
    };
    add(nl++, top.left);
    add(nl++, top.right);
    while (nl < kTreeletLeaves) {
        int pick = -1;
        float largest = -1.0f;
        for (int j = 0; j < nl; ++j) {
            float a = half_area(box[j]);
            if (expandable[j] && a > largest) {
                largest = a;
                pick = j;
            }
        }
        if (pick < 0) break;
        BvhBinaryNode x = load_node(nodes, leaf[pick]);
        inner[ni++] = leaf[pick];
        old_cost += half_area(x.box);
        add(pick, x.left);
        add(nl++, x.right);
    }
    for (int j = 0; j < nl; ++j) old_cost += sub[j];
    if (nl < 3) return old_cost;  // one topology only
    float area[kTreeletSubsets], best[kTreeletSubsets];
    uint8_t split[kTreeletSubsets];
    const int full = (1 << nl) - 1;
    for (int s = 1; s <= full; ++s) {
        int low = __ffs(s) - 1;
        BvhBox u = box[low];
        for (int j = low + 1; j < nl; ++j)
            if (s & (1 << j)) u = merged(u, box[j]);
        area[s] = half_area(u);
        if ((s & (s - 1)) == 0) {
            best[s] = sub[low];
            split[s] = 0;
            continue;
        }
        float b = INFINITY;
        int bq = 0;
        for (int q = (s - 1) & s; q > 0; q = (q - 1) & s) {
            if (!(q & (1 << low))) continue;  // each split once: the side holding the lowest leaf
            float c = best[q] + best[s ^ q];
            if (c < b) {
                b = c;
                bq = q;
            }
        }
        best[s] = area[s] + b;
        split[s] = uint8_t(bq);
    }
    // Keep the current treelet unless the new one is clearly cheaper (the two
    // sums round differently).
    if (!(best[full] < old_cost * (1.0f - 1e-5f))) return old_cost;
    // A finite best cost implies a proper split at every set of the chosen
    // topology; check that before writing anything (non-finite boxes).
    int set_stack[kTreeletLeaves];
    {
        int n_sets = 0, pending = 0;
        set_stack[pending++] = full;
        while (pending > 0) {
            int s = set_stack[--pending];
            int q = split[s];
            if (q == 0 || (q & ~s) != 0 || q == s || ++n_sets > kTreeletLeaves - 1) return old_cost;
            int sides[2] = {q, s ^ q};
            for (int k = 0; k < 2; ++k)
                if ((sides[k] & (sides[k] - 1)) != 0) set_stack[pending++] = sides[k];
        }
    }
    uint32_t node_stack[kTreeletLeaves];
    int top_at = 0, next_inner = 1;
    set_stack[top_at] = full;
    node_stack[top_at++] = root;
    while (top_at > 0) {
        --top_at;
        int s = set_stack[top_at];
        uint32_t slot = node_stack[top_at];
        int sides[2] = {split[s], s ^ split[s]};
        uint32_t child[2];
        for (int k = 0; k < 2; ++k) {
            int t = sides[k];
            if ((t & (t - 1)) == 0) {
                child[k] = leaf[__ffs(t) - 1];
            } else {
                child[k] = inner[next_inner++];
                set_stack[top_at] = t;
                node_stack[top_at++] = child[k];
            }
        }
        int low = __ffs(s) - 1;
        BvhBox u = box[low];
        uint32_t leaves = 0;
        for (int j = low; j < nl; ++j) {
            if (!(s & (1 << j))) continue;
            u = merged(u, box[j]);
            leaves += count[j];
        }
        store_node(nodes, slot, u, child[0], child[1]);
        __stcg(parent + child[0], slot);
        __stcg(parent + child[1], slot);
        __stcg(cost + slot, best[s]);
        __stcg(leafcount + slot, leaves);
    }
    return best[full];
}

// One bottom-up round: thread i starts at leaf i.
__global__ void __launch_bounds__(kRestructureThreads) k_restructure(BvhBinaryNode* nodes, uint32_t* parent,
                                                                     uint32_t* visits, float* cost,
                                                                     uint32_t* leafcount, uint32_t n,
                                                                     uint32_t min_leaves) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    for (uint32_t step = 0; step < 2 * n; ++step) {  // a path to the root is shorter than the node count
        uint32_t p = __ldcg(parent + v);
        if (p == kInvalidChild) return;
        __threadfence();  // this subtree's writes before the arrival
        if (atomicAdd(visits + p, 1u) == 0u) return;  // the other subtree is still being built
        __threadfence();
        BvhBinaryNode node = load_node(nodes, p);
        uint32_t leaves = __ldcg(leafcount + node.left) + __ldcg(leafcount + node.right);
        float c = leaves >= min_leaves ? optimize_treelet(nodes, parent, cost, leafcount, p, node)
                                       : half_area(node.box) + __ldcg(cost + node.left) + __ldcg(cost + node.right);
        __stcg(cost + p, c);
        __stcg(leafcount + p, leaves);
        v = p;
    }
}

// Longest leaf-to-root path; depth[1] is set if a walk does not reach the
// root within the node count (a broken parent chain).
__global__ void k_tree_depth(const uint32_t* parent, uint32_t n, uint32_t* depth) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    uint32_t d = 0;
    while (true) {
        uint32_t p = parent[v];
        if (p == kInvalidChild) break;
        if (++d >= 2 * n) {
            atomicOr(depth + 1, 1u);
            return;
        }
        v = p;
    }
    atomicMax(depth, d);
}

// ------------------------------------------------ top-level rebuild
// The restructured tree is cut into clusters, the largest subtrees with at
// most kTopClusterLeaves leaves; the host's binned-SAH builder rebuilds the
// tree above them, whose n_c - 1 internal nodes take the slots of the n_c - 1
// nodes above the cut.  Treelets cannot see past 7 leaves, and a full SAH
// sweep over ~n/10 clusters costs a fraction of one over n primitives.
constexpr uint32_t kTopClusterLeaves = 16;

__global__ void k_cut_flags(const uint32_t* parent, const uint32_t* leafcount, uint32_t node_count, uint32_t limit,
                            uint32_t* is_cut, uint32_t* is_top) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= node_count) return;
    uint32_t leaves = leafcount[v], p = parent[v];
    is_top[v] = leaves > limit ? 1u : 0u;
    is_cut[v] = leaves <= limit && (p == kInvalidChild || leafcount[p] > limit) ? 1u : 0u;
}

__global__ void k_compact(const uint32_t* flag, const uint32_t* at, uint32_t count, uint32_t* out) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < count && flag[v]) out[at[v]] = v;
}

// Height of every cluster (longest path from it down to a leaf); error[0] is
// set if a leaf has no cluster above it.
__global__ void k_cut_heights(const uint32_t* parent, const uint32_t* is_cut, const uint32_t* cut_at, uint32_t n,
                              uint32_t* height, uint32_t* error) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    uint32_t d = 0;
    while (!is_cut[v]) {
        v = parent[v];
        if (v == kInvalidChild || ++d >= 2 * n) {
            atomicOr(error, 1u);
            return;
        }
    }
    atomicMax(height + cut_at[v], d);
}

// Device -> host.  Large copies go through two pinned staging buffers, so
// the copy of one chunk overlaps the host copy of the previous one (fresh
// pageable memory would otherwise take the transfer through page faults);
// small ones are not worth pinning the buffers (~40 ms).
cudaError_t download(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    constexpr size_t kChunk = size_t(32) << 20;
    if (bytes == 0) return cudaSuccess;
    if (bytes < 4 * kChunk) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
        return e ? e : cudaStreamSynchronize(st);
    }
    void* staging[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && !e; ++k) {
        e = cudaMallocHost(&staging[k], kChunk);
        if (!e) e = cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming);
    }
    size_t chunks = (bytes + kChunk - 1) / kChunk;
    for (size_t c = 0; c < chunks + 1 && !e; ++c) {
        if (c < chunks) {  // start chunk c
            size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
            e = cudaMemcpyAsync(staging[c & 1], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, st);
            if (!e) e = cudaEventRecord(done[c & 1], st);
        }
        if (c > 0 && !e) {  // finish chunk c - 1
            size_t p = c - 1, off = p * kChunk, len = std::min(kChunk, bytes - off);
            e = cudaEventSynchronize(done[p & 1]);
            if (!e) std::memcpy(static_cast<char*>(dst) + off, staging[p & 1], len);
        }
    }
    for (int k = 0; k < 2; ++k) {
        if (done[k]) cudaEventDestroy(done[k]);
        if (staging[k]) cudaFreeHost(staging[k]);
    }
    return e;
}

uint32_t blocks_for(uint32_t n, uint32_t threads) { return (n + threads - 1) / threads; }

// Replaces the nodes above the clusters with the host builder's tree over
// the clusters' boxes: its root takes the root's slot (the last node), its
// other internal nodes the remaining slots in order.  Skipped, keeping the
// tree as it is, if the result would be deeper than `max_depth`.
void rebuild_top(std::vector<BvhBinaryNode>& nodes, const std::vector<uint32_t>& clusters,
                 const std::vector<uint32_t>& cluster_height, const std::vector<uint32_t>& top_slots,
                 int max_depth, int threads) {
    const uint32_t root_slot = uint32_t(nodes.size() - 1);
    std::vector<BvhBox> boxes(clusters.size());
    for (size_t k = 0; k < clusters.size(); ++k) boxes[k] = nodes[clusters[k]].box;
    std::vector<BvhBinaryNode> top;
    build_binary_bvh(boxes.data(), uint32_t(boxes.size()), top, threads);
    if (top.size() != 2 * clusters.size() - 1) return;
    // depth of every cluster in the new top tree plus its own height
    std::vector<std::pair<uint32_t, uint32_t>> stack{{uint32_t(top.size() - 1), 0u}};
    uint32_t deepest = 0;
    while (!stack.empty()) {
        auto [k, d] = stack.back();
        stack.pop_back();
        if (top[k].left == kInvalidChild) {
            deepest = std::max(deepest, d + cluster_height[top[k].right]);
            continue;
        }
        stack.push_back({top[k].left, d + 1});
        stack.push_back({top[k].right, d + 1});
    }
    if (int(deepest) > max_depth) return;
    std::vector<uint32_t> slot(top.size(), kInvalidChild);
    size_t next = 0;
    for (size_t k = 0; k + 1 < top.size(); ++k) {
        if (top[k].left == kInvalidChild) continue;
        while (next < top_slots.size() && top_slots[next] == root_slot) ++next;
        if (next == top_slots.size()) return;
        slot[k] = top_slots[next++];
    }
    slot[top.size() - 1] = root_slot;
    auto ref = [&](uint32_t k) { return top[k].left == kInvalidChild ? clusters[top[k].right] : slot[k]; };
    for (size_t k = 0; k < top.size(); ++k)
        if (top[k].left != kInvalidChild)
            nodes[slot[k]] = BvhBinaryNode{top[k].box, ref(top[k].left), ref(top[k].right)};
}

}  // namespace

bool build_binary_bvh_gpu(const BvhBox* prims, uint32_t n, std::vector<BvhBinaryNode>& out, int max_depth,
                          char* why, size_t why_size, int threads) {
    auto failed = [&](const char* what, cudaError_t e) {
        if (why && why_size) std::snprintf(why, why_size, "%s: %s", what, cudaGetErrorString(e));
        return false;
    };
    out.clear();
    if (n == 0) return true;
    cudaStream_t st = nullptr;
    if (cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) return failed("cudaStreamCreate", e);
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    Scratch scratch;
    const uint32_t node_count = 2 * n - 1;
    BvhBox* d_prims = scratch.alloc<BvhBox>(n);
    BvhBinaryNode* d_nodes = scratch.alloc<BvhBinaryNode>(node_count);
    unsigned long long* keys[2] = {scratch.alloc<unsigned long long>(n), scratch.alloc<unsigned long long>(n)};
    uint32_t* values[2] = {scratch.alloc<uint32_t>(n), scratch.alloc<uint32_t>(n)};
    uint32_t sort_blocks = blocks_for(n, kSortTile);
    uint32_t* hist = scratch.alloc<uint32_t>(size_t(sort_blocks) * 256);
    uint32_t* hist_at = scratch.alloc<uint32_t>(size_t(sort_blocks) * 256);
    uint32_t* bounds = scratch.alloc<uint32_t>(6);
    uint32_t* clusters[2] = {scratch.alloc<uint32_t>(n), scratch.alloc<uint32_t>(n)};
    BvhBox* boxes[2] = {scratch.alloc<BvhBox>(n), scratch.alloc<BvhBox>(n)};
    uint32_t* nearest = scratch.alloc<uint32_t>(n);
    uint32_t* alive = scratch.alloc<uint32_t>(n);
    uint32_t* alive_at = scratch.alloc<uint32_t>(n);
    uint32_t* leader = scratch.alloc<uint32_t>(n);
    uint32_t* leader_at = scratch.alloc<uint32_t>(n);
    if (scratch.error != cudaSuccess) return failed("device memory for the BVH build", scratch.error);
    cudaError_t e = cudaMemcpyAsync(d_prims, prims, sizeof(BvhBox) * n, cudaMemcpyHostToDevice, st);
    uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    if (!e) e = cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e) return failed("BVH input upload", e);

    k_centroid_bounds<<<std::min(blocks_for(n, 256), 4096u), 256, 0, st>>>(d_prims, n, bounds);
    k_morton<<<blocks_for(n, 256), 256, 0, st>>>(d_prims, n, bounds, keys[0], values[0]);
    if ((e = cudaGetLastError())) return failed("Morton keys", e);
    int cur = 0;
    for (int shift = 0; shift < 64; shift += 8) {
        k_sort_histogram<<<sort_blocks, kSortThreads, 0, st>>>(keys[cur], n, shift, hist);
        if ((e = exclusive_scan(hist, hist_at, sort_blocks * 256, st, scratch))) return failed("sort scan", e);
        k_sort_scatter<<<sort_blocks, kSortThreads, 0, st>>>(keys[cur], values[cur], n, shift, hist_at,
                                                             keys[cur ^ 1], values[cur ^ 1]);
        if ((e = cudaGetLastError())) return failed("sort scatter", e);
        cur ^= 1;
    }
    k_leaves<<<blocks_for(n, 256), 256, 0, st>>>(d_prims, values[cur], n, d_nodes, clusters[0], boxes[0]);
    if ((e = cudaGetLastError())) return failed("PLOC leaves", e);

    uint32_t m = n, node_base = n;
    int c = 0, rounds = 0;
    while (m > 1) {
        if (++rounds > kMaxRounds) {  // far beyond the ~log(n) rounds PLOC takes: leave it to the host builder
            if (why && why_size) std::snprintf(why, why_size, "PLOC exceeded %d rounds", kMaxRounds);
            return false;
        }
        k_nearest<<<blocks_for(m, kNearestThreads), kNearestThreads, 0, st>>>(boxes[c], m, nearest);
        k_merge_flags<<<blocks_for(m, 256), 256, 0, st>>>(nearest, m, alive, leader);
        if ((e = cudaGetLastError())) return failed("PLOC neighbours", e);
        if ((e = exclusive_scan(alive, alive_at, m, st, scratch))) return failed("PLOC scan", e);
        if ((e = exclusive_scan(leader, leader_at, m, st, scratch))) return failed("PLOC scan", e);
        k_merge<<<blocks_for(m, 256), 256, 0, st>>>(clusters[c], boxes[c], nearest, m, alive, alive_at, leader,
                                                    leader_at, node_base, d_nodes, clusters[c ^ 1], boxes[c ^ 1]);
        if ((e = cudaGetLastError())) return failed("PLOC merge", e);
        uint32_t tail[4];
        e = cudaMemcpyAsync(&tail[0], alive_at + m - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(&tail[1], alive + m - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(&tail[2], leader_at + m - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(&tail[3], leader + m - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) return failed("PLOC round", e);
        uint32_t survivors = tail[0] + tail[1], merges = tail[2] + tail[3];
        if (merges == 0 || survivors + merges != m) {  // a round always merges the closest pair
            if (why && why_size) std::snprintf(why, why_size, "PLOC made no progress at %u clusters", m);
            return false;
        }
        node_base += merges;
        m = survivors;
        c ^= 1;
    }
    uint32_t depth = 0;
    std::vector<uint32_t> top_clusters, cluster_height, top_slots;  // top-level rebuild (empty: none)
    if (n >= 2) {
        // Treelet restructuring; it may change the depth, which is measured
        // afterwards.
        uint32_t* parent = scratch.alloc<uint32_t>(node_count);
        uint32_t* visits = scratch.alloc<uint32_t>(node_count);
        uint32_t* leafcount = scratch.alloc<uint32_t>(node_count);
        float* cost = scratch.alloc<float>(node_count);
        uint32_t* d_depth = scratch.alloc<uint32_t>(2);
        if (scratch.error != cudaSuccess) return failed("device memory for the BVH restructuring", scratch.error);
        e = cudaMemsetAsync(parent + node_count - 1, 0xff, sizeof(uint32_t), st);
        if (!e) e = cudaMemsetAsync(d_depth, 0, 2 * sizeof(uint32_t), st);
        if (e) return failed("BVH restructuring setup", e);
        k_parents<<<blocks_for(n - 1, 256), 256, 0, st>>>(d_nodes, n, parent);
        k_leaf_costs<<<blocks_for(n, 256), 256, 0, st>>>(d_nodes, n, cost, leafcount);
        if ((e = cudaGetLastError())) return failed("BVH parents", e);
        for (int round = 0; round < kRestructureRounds; ++round) {
            if ((e = cudaMemsetAsync(visits, 0, sizeof(uint32_t) * node_count, st))) return failed("BVH visits", e);
            k_restructure<<<blocks_for(n, kRestructureThreads), kRestructureThreads, 0, st>>>(
                d_nodes, parent, visits, cost, leafcount, n, uint32_t(kTreeletLeaves) << round);
            if ((e = cudaGetLastError())) return failed("BVH treelet restructuring", e);
        }
        k_tree_depth<<<blocks_for(n, 256), 256, 0, st>>>(parent, n, d_depth);
        uint32_t result[2] = {0, 0};
        e = cudaMemcpyAsync(result, d_depth, sizeof(result), cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) return failed("BVH depth", e);
        if (result[1]) {
            if (why && why_size) std::snprintf(why, why_size, "restructured BVH has a broken parent chain");
            return false;
        }
        depth = result[0];
        // Clusters of the top-level rebuild, their heights and the slots
        // above them.
        uint32_t* is_cut = scratch.alloc<uint32_t>(node_count);
        uint32_t* is_top = scratch.alloc<uint32_t>(node_count);
        uint32_t* cut_at = scratch.alloc<uint32_t>(node_count);
        uint32_t* top_at = scratch.alloc<uint32_t>(node_count);
        if (scratch.error != cudaSuccess) return failed("device memory for the BVH top rebuild", scratch.error);
        k_cut_flags<<<blocks_for(node_count, 256), 256, 0, st>>>(parent, leafcount, node_count, kTopClusterLeaves,
                                                                 is_cut, is_top);
        if ((e = cudaGetLastError())) return failed("BVH clusters", e);
        if ((e = exclusive_scan(is_cut, cut_at, node_count, st, scratch))) return failed("BVH cluster scan", e);
        if ((e = exclusive_scan(is_top, top_at, node_count, st, scratch))) return failed("BVH cluster scan", e);
        uint32_t tail[4];
        e = cudaMemcpyAsync(&tail[0], cut_at + node_count - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(&tail[1], is_cut + node_count - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(&tail[2], top_at + node_count - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(&tail[3], is_top + node_count - 1, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) return failed("BVH cluster counts", e);
        uint32_t clusters_n = tail[0] + tail[1], top_n = tail[2] + tail[3];
        if (clusters_n >= 3 && top_n == clusters_n - 1) {
            uint32_t* cut_list = scratch.alloc<uint32_t>(clusters_n);
            uint32_t* top_list = scratch.alloc<uint32_t>(top_n);
            uint32_t* cut_height = scratch.alloc<uint32_t>(clusters_n);
            if (scratch.error != cudaSuccess) return failed("device memory for the BVH top rebuild", scratch.error);
            if ((e = cudaMemsetAsync(cut_height, 0, sizeof(uint32_t) * clusters_n, st)) ||
                (e = cudaMemsetAsync(d_depth + 1, 0, sizeof(uint32_t), st)))
                return failed("BVH cluster heights", e);
            k_compact<<<blocks_for(node_count, 256), 256, 0, st>>>(is_cut, cut_at, node_count, cut_list);
            k_compact<<<blocks_for(node_count, 256), 256, 0, st>>>(is_top, top_at, node_count, top_list);
            k_cut_heights<<<blocks_for(n, 256), 256, 0, st>>>(parent, is_cut, cut_at, n, cut_height, d_depth + 1);
            if ((e = cudaGetLastError())) return failed("BVH cluster heights", e);
            top_clusters.resize(clusters_n);
            cluster_height.resize(clusters_n);
            top_slots.resize(top_n);
            uint32_t broken = 0;
            e = cudaMemcpyAsync(top_clusters.data(), cut_list, 4 * size_t(clusters_n), cudaMemcpyDeviceToHost, st);
            if (!e) e = cudaMemcpyAsync(cluster_height.data(), cut_height, 4 * size_t(clusters_n),
                                        cudaMemcpyDeviceToHost, st);
            if (!e) e = cudaMemcpyAsync(top_slots.data(), top_list, 4 * size_t(top_n), cudaMemcpyDeviceToHost, st);
            if (!e) e = cudaMemcpyAsync(&broken, d_depth + 1, 4, cudaMemcpyDeviceToHost, st);
            if (!e) e = cudaStreamSynchronize(st);
            if (e) return failed("BVH clusters download", e);
            if (broken) top_clusters.clear();  // keep the restructured tree
        }
    }
    if (int(depth) > max_depth) {
        if (why && why_size) std::snprintf(why, why_size, "GPU BVH depth %u exceeds %d", depth, max_depth);
        return false;
    }
    // Leaves are known on the host (box i, primitive i); only the n-1
    // internal nodes come back.
    out.resize(node_count);
    for (uint32_t i = 0; i < n; ++i) out[i] = BvhBinaryNode{prims[i], kInvalidChild, i};
    e = download(out.data() + n, d_nodes + n, sizeof(BvhBinaryNode) * (node_count - n), st);
    if (e) {
        out.clear();
        return failed("BVH download", e);
    }
    if (!top_clusters.empty()) rebuild_top(out, top_clusters, cluster_height, top_slots, max_depth, threads);
    return true;
}

}  // namespace wf
