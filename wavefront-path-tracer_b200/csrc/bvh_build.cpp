// Binned-SAH binary BVH builder.  See bvh_build.h for the output contract.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>

namespace wf {
namespace {

constexpr int kBins = 32;
constexpr uint32_t kParallelThreshold = 32768;

inline float half_area(const BvhBox& b) {
    float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

inline void grow(BvhBox& b, const BvhBox& o) {
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(b.lo[a], o.lo[a]);
        b.hi[a] = std::max(b.hi[a], o.hi[a]);
    }
}

inline BvhBox empty_box() {
    BvhBox b;
    for (int a = 0; a < 3; ++a) { b.lo[a] = INFINITY; b.hi[a] = -INFINITY; }
    return b;
}

inline int ceil_log2(uint32_t n) {
    int r = 0;
    while ((1ull << r) < n) ++r;
    return r;
}

struct Builder {
    const BvhBox* prims;
    std::vector<float> centroid;   // 3 per primitive
    std::vector<uint32_t> index;
    BvhBinaryNode* nodes;
    std::atomic<int> spare_threads;

    float c(uint32_t prim, int axis) const { return centroid[3 * size_t(prim) + axis]; }

    uint32_t median_split(uint32_t begin, uint32_t end, int axis) {
        uint32_t mid = begin + (end - begin) / 2;
        std::nth_element(index.begin() + begin, index.begin() + mid, index.begin() + end,
            [&](uint32_t a, uint32_t b) {
                float ca = c(a, axis), cb = c(b, axis);
                return ca < cb || (ca == cb && a < b);
            });
        return mid;
    }

    uint32_t choose_split(uint32_t begin, uint32_t end, int depth) {
        uint32_t n = end - begin;
        float cmin[3] = {INFINITY, INFINITY, INFINITY};
        float cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = begin; i < end; ++i) {
            uint32_t p = index[i];
            for (int a = 0; a < 3; ++a) {
                cmin[a] = std::min(cmin[a], c(p, a));
                cmax[a] = std::max(cmax[a], c(p, a));
            }
        }
        int widest = 0;
        for (int a = 1; a < 3; ++a)
            if (cmax[a] - cmin[a] > cmax[widest] - cmin[widest]) widest = a;
        if (!(cmax[widest] - cmin[widest] > 0.0f))
            return begin + n / 2;  // all centroids coincide: any split is equal
        if (depth + ceil_log2(n) >= kMaxBvhDepth || n <= 2)
            return median_split(begin, end, widest);

        float best_cost = INFINITY;
        int best_axis = -1, best_bin = -1;
        for (int a = 0; a < 3; ++a) {
            float extent = cmax[a] - cmin[a];
            if (!(extent > 0.0f)) continue;
            float scale = float(kBins) / extent;
            BvhBox bin_box[kBins];
            uint32_t bin_count[kBins];
            for (int b = 0; b < kBins; ++b) { bin_box[b] = empty_box(); bin_count[b] = 0; }
            for (uint32_t i = begin; i < end; ++i) {
                uint32_t p = index[i];
                int b = std::min(kBins - 1, int((c(p, a) - cmin[a]) * scale));
                grow(bin_box[b], prims[p]);
                ++bin_count[b];
            }
            float right_area[kBins];
            uint32_t right_count[kBins];
            BvhBox acc = empty_box();
            uint32_t cnt = 0;
            for (int b = kBins - 1; b > 0; --b) {
                if (bin_count[b]) grow(acc, bin_box[b]);
                cnt += bin_count[b];
                right_area[b] = cnt ? half_area(acc) : 0.0f;
                right_count[b] = cnt;
            }
            acc = empty_box();
            cnt = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                if (bin_count[b]) grow(acc, bin_box[b]);
                cnt += bin_count[b];
                if (cnt == 0 || right_count[b + 1] == 0) continue;
                float cost = half_area(acc) * float(cnt) + right_area[b + 1] * float(right_count[b + 1]);
                if (cost < best_cost) { best_cost = cost; best_axis = a; best_bin = b; }
            }
        }
        if (best_axis < 0)
            return median_split(begin, end, widest);
        float scale = float(kBins) / (cmax[best_axis] - cmin[best_axis]);
        float lo = cmin[best_axis];
        auto it = std::partition(index.begin() + begin, index.begin() + end, [&](uint32_t p) {
            return std::min(kBins - 1, int((c(p, best_axis) - lo) * scale)) <= best_bin;
        });
        uint32_t mid = uint32_t(it - index.begin());
        if (mid == begin || mid == end)
            return median_split(begin, end, widest);
        return mid;
    }

    // Builds prims index[begin, end) into nodes [base, base + 2n - 1); root last.
    void build(uint32_t begin, uint32_t end, uint32_t base, int depth) {
        uint32_t n = end - begin;
        if (n == 1) {
            uint32_t p = index[begin];
            nodes[base] = BvhBinaryNode{prims[p], kInvalidChild, p};
            return;
        }
        uint32_t mid = choose_split(begin, end, depth);
        uint32_t nl = mid - begin, nr = end - mid;
        uint32_t left_base = base, right_base = base + 2 * nl - 1;
        uint32_t left_root = left_base + 2 * nl - 2, right_root = right_base + 2 * nr - 2;
        bool spawned = false;
        std::thread worker;
        if (n >= kParallelThreshold && nl >= 1024 && spare_threads.fetch_sub(1) > 0) {
            spawned = true;
            worker = std::thread([=] { build(begin, mid, left_base, depth + 1); });
        } else if (n >= kParallelThreshold && nl >= 1024) {
            spare_threads.fetch_add(1);
        }
        if (!spawned) build(begin, mid, left_base, depth + 1);
        build(mid, end, right_base, depth + 1);
        if (spawned) {
            worker.join();
            spare_threads.fetch_add(1);
        }
        BvhBox box = nodes[left_root].box;
        grow(box, nodes[right_root].box);
        nodes[base + 2 * n - 2] = BvhBinaryNode{box, left_root, right_root};
    }
};

int depth_of(const std::vector<BvhBinaryNode>& nodes, uint32_t node, int depth) {
    const BvhBinaryNode& x = nodes[node];
    if (x.left == kInvalidChild) return depth;
    return std::max(depth_of(nodes, x.left, depth + 1), depth_of(nodes, x.right, depth + 1));
}

}  // namespace

void build_binary_bvh(const BvhBox* prims, uint32_t count,
                      std::vector<BvhBinaryNode>& nodes, int threads) {
    nodes.clear();
    if (count == 0) return;
    nodes.resize(2 * size_t(count) - 1);
    Builder b;
    b.prims = prims;
    b.nodes = nodes.data();
    b.centroid.resize(3 * size_t(count));
    b.index.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        b.index[i] = i;
        for (int a = 0; a < 3; ++a)
            b.centroid[3 * size_t(i) + a] = (prims[i].lo[a] + prims[i].hi[a]) * 0.5f;
    }
    if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
    b.spare_threads = threads - 1;
    b.build(0, count, 0, 0);
}

int binary_bvh_depth(const std::vector<BvhBinaryNode>& nodes) {
    if (nodes.empty()) return 0;
    return depth_of(nodes, uint32_t(nodes.size() - 1), 0);
}

}  // namespace wf
