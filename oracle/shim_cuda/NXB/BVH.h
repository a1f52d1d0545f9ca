// Project-written stand-in for the NexusBVH types, for the reference's CUDA
// renderer built for sm_100a (oracle/Makefile, target `cuda`).
//
// ORACLE / TEST INFRASTRUCTURE ONLY.  NexusBVH (https://github.com/StokastX/NexusBVH,
// an un-vendored submodule, .gitmodules:1-3, no commit pinned) is absent from
// the reference tree.  The types are the ones the host shim (oracle/shim/NXB/BVH.h)
// restates from the reference's call sites (include/renderer/device_traversal.cuh:
// 208-313,845-875,916-945, include/scene/scene.cuh:16,131-134,171-177), with
// device storage: a BVH2 owns its node array in device memory, DeviceBuffer
// holds a device copy, and BuildBVH2 (oracle/ref_cuda_harness.cu) reads the
// primitives back, builds with the project's binned-SAH builder on the host
// and uploads the nodes, so this build traverses the same trees as the
// host-compiled reference and the B200 renderer.
#pragma once

#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <vector>

#include <cuda_runtime.h>

namespace NXB {

constexpr uint32_t InvalidIdx = 0xffffffffu;

struct AABB {
    float3 bMin;
    float3 bMax;
    __host__ __device__ AABB()
        : bMin(make_float3(INFINITY, INFINITY, INFINITY)), bMax(make_float3(-INFINITY, -INFINITY, -INFINITY)) {}
    __host__ __device__ AABB(float3 lo, float3 hi) : bMin(lo), bMax(hi) {}
    __host__ __device__ void Clear() {
        bMin = make_float3(INFINITY, INFINITY, INFINITY);
        bMax = make_float3(-INFINITY, -INFINITY, -INFINITY);
    }
};

struct Triangle {
    float3 v0, v1, v2;
    __host__ __device__ Triangle(float3 a, float3 b, float3 c) : v0(a), v1(b), v2(c) {}
};

struct BuildConfig {};

struct BVHBuildMetrics {
    float computeSceneBoundsTime = 0, computeMortonCodesTime = 0, radixSortTime = 0, bvhBuildTime = 0;
};

namespace detail {
struct DeviceFree {
    void operator()(void* p) const {
        if (p) cudaFree(p);
    }
};
template <typename T>
std::shared_ptr<T> device_copy(const T* host, size_t count) {
    if (count == 0) return {};
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * count) != cudaSuccess) throw std::runtime_error("NXB shim: cudaMalloc failed");
    std::shared_ptr<T> owned(static_cast<T*>(p), DeviceFree{});
    if (cudaMemcpy(p, host, sizeof(T) * count, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("NXB shim: cudaMemcpy failed");
    return owned;
}
}  // namespace detail

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
    DeviceView View() const { return DeviceView{nodes_.get(), nodeCount_, primCount_, bounds_}; }
    const AABB& Bounds() const { return bounds_; }
    uint32_t NodeCount() const { return nodeCount_; }

    std::shared_ptr<Node> nodes_;  // device memory, freed with the last copy
    uint32_t nodeCount_ = 0;
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
    explicit DeviceBuffer(const std::vector<T>& values)
        : data_(detail::device_copy(values.data(), values.size())), count_(values.size()) {}
    T* Get() { return data_.get(); }
    size_t Size() const { return count_; }

private:
    std::shared_ptr<T> data_;
    size_t count_;
};

BVH2 BuildBVH2(const Triangle* triangles, uint32_t count, BuildConfig config = {}, BVHBuildMetrics* metrics = nullptr);
BVH2 BuildBVH2(const AABB* boxes, uint32_t count, BuildConfig config = {}, BVHBuildMetrics* metrics = nullptr);
BVH8 BuildBVH8(const Triangle* triangles, uint32_t count, BuildConfig config = {}, BVHBuildMetrics* metrics = nullptr);

}  // namespace NXB
