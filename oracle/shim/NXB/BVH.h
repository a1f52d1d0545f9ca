// Project-written stand-in for the NexusBVH types the reference uses.
//
// ORACLE / TEST INFRASTRUCTURE ONLY.  NexusBVH (https://github.com/StokastX/NexusBVH,
// an un-vendored submodule, .gitmodules:1-3, no commit pinned) is absent from
// the reference tree.  Its types are restated here from the reference's call
// sites: include/renderer/device_traversal.cuh:208-313,845-875,916-945,
// include/scene/scene.cuh:16,131-134,171-177, tests/material_transport_tests.cu:22-26,84-91.
// The builder behind BuildBVH2 is the project's own binned-SAH builder
// (wavefront-path-tracer_b200/csrc/bvh_build.cpp), so the host-compiled
// reference traverses exactly the trees the CUDA renderer traverses.
#pragma once

#include <cstdint>
#include <cmath>
#include <vector>
#include <cuda_runtime.h>

namespace NXB {

constexpr uint32_t InvalidIdx = 0xffffffffu;

struct AABB {
    float3 bMin;
    float3 bMax;
    AABB() : bMin(make_float3(INFINITY, INFINITY, INFINITY)), bMax(make_float3(-INFINITY, -INFINITY, -INFINITY)) {}
    AABB(float3 lo, float3 hi) : bMin(lo), bMax(hi) {}
    void Clear() {
        bMin = make_float3(INFINITY, INFINITY, INFINITY);
        bMax = make_float3(-INFINITY, -INFINITY, -INFINITY);
    }
};

struct Triangle {
    float3 v0, v1, v2;
    Triangle(float3 a, float3 b, float3 c) : v0(a), v1(b), v2(c) {}
};

struct BuildConfig {};

struct BVHBuildMetrics {
    float computeSceneBoundsTime = 0, computeMortonCodesTime = 0, radixSortTime = 0, bvhBuildTime = 0;
};

class BVH2 {
public:
    struct Node {
        AABB bounds;
        uint32_t leftChild;
        uint32_t rightChild;
    };
    struct DeviceView {
        Node* nodes;
        uint32_t nodeCount;
        uint32_t primCount;
        AABB bounds;
    };
    BVH2() = default;
    DeviceView View() const {
        return DeviceView{storage_.empty() ? nullptr : const_cast<Node*>(storage_.data()),
                          uint32_t(storage_.size()), primCount_, bounds_};
    }
    const AABB& Bounds() const { return bounds_; }
    uint32_t NodeCount() const { return uint32_t(storage_.size()); }
    std::vector<Node> storage_;
    uint32_t primCount_ = 0;
    AABB bounds_;
};

class BVH8 {
public:
    struct NodeExplicit {
        float3 p;
        uint8_t e[3];
        uint8_t imask;
        uint32_t childBaseIdx;
        uint32_t primBaseIdx;
        uint8_t meta[8];
        uint8_t qlox[8], qloy[8], qloz[8], qhix[8], qhiy[8], qhiz[8];
    };
    using Node = NodeExplicit;
    struct DeviceView {
        Node* nodes = nullptr;
        uint32_t* primIdx = nullptr;
        uint32_t nodeCount = 0;
        uint32_t primCount = 0;
    };
    DeviceView View() const { return DeviceView{}; }
    uint32_t NodeCount() const { return 0; }
    float AverageChildPerNode() const { return 0.0f; }
};

template <typename T>
class DeviceBuffer {
public:
    explicit DeviceBuffer(const std::vector<T>& values) : values_(values) {}
    T* Get() { return values_.data(); }
private:
    std::vector<T> values_;
};

BVH2 BuildBVH2(const Triangle* triangles, uint32_t count, BuildConfig config = {}, BVHBuildMetrics* metrics = nullptr);
BVH2 BuildBVH2(const AABB* boxes, uint32_t count, BuildConfig config = {}, BVHBuildMetrics* metrics = nullptr);
BVH8 BuildBVH8(const Triangle* triangles, uint32_t count, BuildConfig config = {}, BVHBuildMetrics* metrics = nullptr);

}  // namespace NXB
