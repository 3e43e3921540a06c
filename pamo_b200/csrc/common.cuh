// Shared definitions for the pamo_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/pamo_b200.h"

namespace pamo {

constexpr int kThreads = 256;
constexpr int kNumSMs = 148;

// Grid for a grid-stride loop over n items: at most 8 resident blocks per SM.
inline int grid_for(long long n, int threads = kThreads)
{
    long long b = (n + threads - 1) / threads;
    long long cap = (long long)kNumSMs * 8;
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

// Every kernel this library starts goes through launch(): it counts the launches
// (pamo_launch_count) and then issues the launch on the given stream.
inline std::atomic<long long> g_launches{0};

// Per-call scratch comes from the device's default stream-ordered pool.  By
// default the pool hands its memory back at every synchronisation, so each
// call would map fresh memory; this keeps up to kPoolKeepBytes in the pool
// (raising the threshold only, never lowering one set by the application).
constexpr unsigned long long kPoolKeepBytes = 1ULL << 30;
inline cudaError_t retain_pool_memory()
{
    static std::atomic<unsigned long long> done{0};  // one bit per device ordinal below 64
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && ((done.load() >> dev) & 1ULL)) return cudaSuccess;
    cudaMemPool_t pool;
    if ((e = cudaDeviceGetDefaultMemPool(&pool, dev)) != cudaSuccess) return e;
    unsigned long long cur = 0;  // the attribute is a 64-bit unsigned value
    if ((e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur)) != cudaSuccess) return e;
    if (cur < kPoolKeepBytes) {
        unsigned long long keep = kPoolKeepBytes;
        if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    }
    if (dev < 64) done.fetch_or(1ULL << dev);
    return cudaSuccess;
}

template <typename... KArgs, typename... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args)
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
    kernel<<<grid, block, smem, s>>>(args...);
}

#define PAMO_CUDA_TRY(expr)                                      \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return pamo::map_cuda_error(_e); \
    } while (0)

inline int map_cuda_error(cudaError_t e)
{
    if (e == cudaErrorMemoryAllocation) return PAMO_ERR_OOM;
    return PAMO_ERR_DEVICE;
}

#define PAMO_GRID_STRIDE(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)(n); i += (long long)blockDim.x * gridDim.x)

// ---------------------------------------------------------------------------
// Arithmetic that must round exactly like the reference kernels
// (simp_cuda/src/cusimp_free.h Vertex<float>/Mat4x4<float>, cusimp_free.cu).
// Everything in this library that feeds a collapse or intersection decision is
// compiled with --fmad=false, so each expression below is evaluated with one
// IEEE rounding per operation, in the written order.
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 v3(float4 p) { return {p.x, p.y, p.z}; }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 vcross(V3 a, V3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float vnorm(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ V3 vdivs(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 vmid(V3 a, V3 b) { return {(a.x + b.x) / 2.0f, (a.y + b.y) / 2.0f, (a.z + b.z) / 2.0f}; }

// the reference's min/max/clamp templates (cusimp_free.cu:29-34): NaN-propagating
// in the same way (a comparison that fails returns the second operand).
__device__ __forceinline__ float tmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float tmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float tclamp(float x, float a, float b) { return tmin(tmax(a, x), b); }

__device__ __forceinline__ bool face_dead(int4 t) { return t.x == -1 && t.y == -1 && t.z == -1; }
__device__ __forceinline__ bool face_has(int4 t, int v) { return t.x == v || t.y == v || t.z == v; }

// sortable encoding of floats for atomicMin/atomicMax on int
__device__ __forceinline__ int float_to_ordered(float f)
{
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float ordered_to_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

}  // namespace pamo
