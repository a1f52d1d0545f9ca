// ORACLE / TEST INFRASTRUCTURE ONLY.  Host stand-in for <cooperative_groups.h>
// so src/renderer/renderer.cu compiles as host C++.  A host "grid" is one
// worker thread, so sync() has nothing to wait for; the persistent kernel is
// only ever run with gridDim = blockDim = 1 on the host.
#pragma once
namespace cooperative_groups {
struct grid_group {
    void sync() const {}
};
inline grid_group this_grid() { return grid_group{}; }
}  // namespace cooperative_groups
