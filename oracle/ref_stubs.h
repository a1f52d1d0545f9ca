// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Force-included (after cuda_runtime.h) when the reference's CUDA sources are
// compiled as host C++ into oracle/_ref/libwfref.so.  It supplies host
// versions of the few CUDA device built-ins the reference uses and routes the
// CUDA runtime calls of src/scene/scene.cu, src/renderer/render_session.cu and
// src/renderer/render_checkpoint.cpp to host memory.  This follows the
// reference's own CPU replay recipe (docs/diagnostics/bmw-hdr-fireflies/
// cpu_replay.cpp:11-26, run_glass_checks.py:20-26): the kernels run unmodified,
// one host thread standing in for one CUDA thread.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

using std::isfinite;
using std::max;
using std::min;

// One host worker = one CUDA thread: each worker sets blockIdx.x to the
// linear thread index with blockDim.x = 1 and threadIdx.x = 0, so every
// "warp" has a single lane.
struct WfRefDim3 {
    unsigned x = 0, y = 0, z = 0;
};
extern thread_local WfRefDim3 blockIdx, blockDim, threadIdx, gridDim;

inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline unsigned __activemask() { return 1u; }
inline unsigned __ballot_sync(unsigned, int predicate) { return predicate ? 1u : 0u; }
template <typename T>
inline T __shfl_sync(unsigned, T value, int) { return value; }
inline unsigned atomicAdd(unsigned* address, unsigned value) {
    return __atomic_fetch_add(address, value, __ATOMIC_RELAXED);
}
inline unsigned atomicExch(unsigned* address, unsigned value) {
    return __atomic_exchange_n(address, value, __ATOMIC_RELAXED);
}

// ---------------------------------------------------------------- textures
// Completes the runtime's opaque array type with a host image.
struct cudaArray {
    uint32_t width = 0, height = 0;
    cudaChannelFormatDesc desc{};
    size_t texelBytes = 0;
    std::vector<unsigned char> data;
};

// Bilinear lookup with the exact arithmetic of the reference's CPU replay
// (cpu_replay.cpp:14-24): texel-centre offset, floor, wrap or clamp per axis,
// weights (1-f, f), accumulated rows then columns.
float4 wfref_texture_fetch(cudaTextureObject_t object, float u, float v);
template <typename T>
T tex2D(cudaTextureObject_t object, float u, float v);
template <>
inline float4 tex2D<float4>(cudaTextureObject_t object, float u, float v) {
    return wfref_texture_fetch(object, u, v);
}

// ----------------------------------------------------------- runtime calls
template <typename T>
inline cudaError_t wfref_cudaMalloc(T** pointer, size_t bytes) {
    *pointer = static_cast<T*>(std::malloc(bytes ? bytes : 1));
    return *pointer ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t wfref_cudaFree(void* pointer) { std::free(pointer); return cudaSuccess; }
inline cudaError_t wfref_cudaMemcpy(void* dst, const void* src, size_t bytes, cudaMemcpyKind) {
    if (bytes) std::memcpy(dst, src, bytes);
    return cudaSuccess;
}
inline cudaError_t wfref_cudaMemcpyAsync(void* dst, const void* src, size_t bytes, cudaMemcpyKind,
                                         cudaStream_t = nullptr) {
    if (bytes) std::memcpy(dst, src, bytes);
    return cudaSuccess;
}
inline cudaError_t wfref_cudaMemset(void* dst, int value, size_t bytes) {
    std::memset(dst, value, bytes);
    return cudaSuccess;
}
inline cudaError_t wfref_cudaMemsetAsync(void* dst, int value, size_t bytes, cudaStream_t = nullptr) {
    std::memset(dst, value, bytes);
    return cudaSuccess;
}
cudaError_t wfref_cudaMallocArray(cudaArray_t* array, const cudaChannelFormatDesc* desc, size_t width,
                                  size_t height, unsigned int flags = 0);
cudaError_t wfref_cudaMemcpy2DToArray(cudaArray_t array, size_t wOffset, size_t hOffset, const void* src,
                                      size_t spitch, size_t width, size_t height, cudaMemcpyKind kind);
cudaError_t wfref_cudaFreeArray(cudaArray_t array);
cudaError_t wfref_cudaCreateTextureObject(cudaTextureObject_t* object, const cudaResourceDesc* resource,
                                          const cudaTextureDesc* texture, const cudaResourceViewDesc* view);
cudaError_t wfref_cudaDestroyTextureObject(cudaTextureObject_t object);
inline const char* wfref_cudaGetErrorString(cudaError_t) { return "host stub error"; }
template <typename T>
inline cudaError_t wfref_cudaHostAlloc(T** pointer, size_t bytes, unsigned int) {
    *pointer = static_cast<T*>(std::malloc(bytes ? bytes : 1));
    return *pointer ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t wfref_cudaFreeHost(void* pointer) { std::free(pointer); return cudaSuccess; }
inline cudaError_t wfref_cudaEventCreateWithFlags(cudaEvent_t* event, unsigned int) {
    *event = nullptr;
    return cudaSuccess;
}
inline cudaError_t wfref_cudaEventRecord(cudaEvent_t, cudaStream_t = nullptr) { return cudaSuccess; }
inline cudaError_t wfref_cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t wfref_cudaEventDestroy(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t wfref_cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
inline cudaError_t wfref_cudaGetLastError() { return cudaSuccess; }
inline cudaError_t wfref_cudaDeviceSynchronize() { return cudaSuccess; }

#define cudaMalloc wfref_cudaMalloc
#define cudaFree wfref_cudaFree
#define cudaMemcpy wfref_cudaMemcpy
#define cudaMemcpyAsync wfref_cudaMemcpyAsync
#define cudaMemset wfref_cudaMemset
#define cudaMemsetAsync wfref_cudaMemsetAsync
#define cudaMallocArray wfref_cudaMallocArray
#define cudaMemcpy2DToArray wfref_cudaMemcpy2DToArray
#define cudaFreeArray wfref_cudaFreeArray
#define cudaCreateTextureObject wfref_cudaCreateTextureObject
#define cudaDestroyTextureObject wfref_cudaDestroyTextureObject
#define cudaGetErrorString wfref_cudaGetErrorString
#define cudaHostAlloc wfref_cudaHostAlloc
#define cudaFreeHost wfref_cudaFreeHost
#define cudaEventCreateWithFlags wfref_cudaEventCreateWithFlags
#define cudaEventRecord wfref_cudaEventRecord
#define cudaEventSynchronize wfref_cudaEventSynchronize
#define cudaEventDestroy wfref_cudaEventDestroy
#define cudaStreamSynchronize wfref_cudaStreamSynchronize
#define cudaGetLastError wfref_cudaGetLastError
#define cudaDeviceSynchronize wfref_cudaDeviceSynchronize
