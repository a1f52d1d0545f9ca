// Binary BVH builder (binned SAH, one primitive per leaf).
//
// Replaces the NexusBVH H-PLOC builder the reference calls at
// src/scene/scene.cu:148-149 (BLAS), :227-228 (TLAS) and :262-264 (direct
// triangles).  The output follows the node semantics the reference traversal
// relies on (include/renderer/device_traversal.cuh:245,254-255):
//   * a leaf has left == kInvalidChild and right == primitive index,
//   * an internal node has left/right = child node indices,
//   * the root is the last node (index 2n-2), children precede parents.
// A tree over n primitives therefore always has exactly 2n-1 nodes, which
// lets subtrees be built in parallel into pre-assigned index ranges: the
// result is identical for any thread count.
#pragma once

#include <cstdint>
#include <vector>

namespace wf {

constexpr uint32_t kInvalidChild = 0xffffffffu;

struct BvhBox {
    float lo[3];
    float hi[3];
};

struct BvhBinaryNode {
    BvhBox box;
    uint32_t left;
    uint32_t right;
};

// Depth of every leaf is kept <= kMaxBvhDepth so a 64-entry traversal stack
// (the reference's maxBvhStackSize, device_traversal.cuh:243,844) never
// overflows: once depth + ceil(log2(n)) reaches the bound the builder switches
// to object-median splits.
constexpr int kMaxBvhDepth = 60;

// Builds the tree over primitive boxes.  `threads` <= 0 uses all hardware
// threads.  Empty input yields an empty node list.
void build_binary_bvh(const BvhBox* prims, uint32_t count,
                      std::vector<BvhBinaryNode>& nodes, int threads = 0);

// Maximum leaf depth (root = 0) of a tree produced above; used by tests.
int binary_bvh_depth(const std::vector<BvhBinaryNode>& nodes);

}  // namespace wf
