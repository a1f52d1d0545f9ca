// GPU BVH2 builder (PLOC), wf_bvh_gpu.cu.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "bvh_build.h"

namespace wf {

// Builds the tree over `count` primitive boxes (host memory) on the current
// device, in the host builder's output format (bvh_build.h), except that after
// the treelet restructuring a child may come after its parent (readers walk
// from the root, the last node).  The levels above subtrees of at most 16
// leaves are rebuilt by the host builder with `threads` threads (<= 0: all
// hardware threads).  Synchronous.
// Returns false with a message in `why` on a CUDA error, a stalled build or a
// leaf deeper than `max_depth` (checked on the device before the download).
bool build_binary_bvh_gpu(const BvhBox* prims, uint32_t count, std::vector<BvhBinaryNode>& nodes, int max_depth,
                          char* why, size_t why_size, int threads = 0);

}  // namespace wf
