// lcs_common.cuh -- shared device helpers for the sm_100a contact-and-solve kernels.
//
// Floating point: the library is compiled with -fmad=false so that nothing is fused behind
// the source's back; every fused multiply-add is written out (__fmaf_rn).  The CPU oracle
// spells out the same operation order, which is what makes the candidate sets, the narrow
// phase filters and the CCD time of impact bit-identical between the two.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lcs_gpu.h"

namespace lcs {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kNumSMs = 148;

struct v3 {
    float x, y, z;
};

__device__ __forceinline__ v3 mk3(float x, float y, float z) { return v3{x, y, z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return v3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return v3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator*(float s, v3 a) { return v3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ v3 neg3(v3 a) { return v3{-a.x, -a.y, -a.z}; }
// dot = fma(z, fma(y, x*x)) -- the oracle's order
__device__ __forceinline__ float dot3(v3 a, v3 b) { return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, a.x * b.x)); }
__device__ __forceinline__ v3 cross3(v3 a, v3 b)
{
    return v3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// min / max as plain selects (same -0 / NaN behaviour as the oracle's)
__device__ __forceinline__ float fmn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ v3 min3(v3 a, v3 b) { return v3{fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z)}; }
__device__ __forceinline__ v3 max3(v3 a, v3 b) { return v3{fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z)}; }

// 16-byte vertex record (LuisaCompute float3 layout)
__device__ __forceinline__ v3 ld3(const float4* __restrict__ x, uint32_t i)
{
    float4 v = __ldg(&x[i]);
    return v3{v.x, v.y, v.z};
}
__device__ __forceinline__ v3 ld3cg(const float4* x, uint32_t i)
{
    float4 v = __ldcg(&x[i]);
    return v3{v.x, v.y, v.z};
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// warp-aggregated append: one atomic per warp per call; returns this lane's slot
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want)
{
    const uint32_t mask = __ballot_sync(__activemask(), want);
    if (!want) return kInvalid;
    const uint32_t leader = __ffs(mask) - 1;
    const uint32_t rank = __popc(mask & ((1u << lane_id()) - 1u));
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + rank;
}

// float min for non-negative values through the integer order of their bit patterns
__device__ __forceinline__ void atomic_min_pos(float* addr, float v)
{
    atomicMin(reinterpret_cast<int*>(addr), __float_as_int(v));
}

inline int grid_for(uint64_t n, int block, int max_blocks_per_sm = 8)
{
    uint64_t g = (n + block - 1) / block;
    uint64_t cap = (uint64_t)kNumSMs * max_blocks_per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace lcs

#define LCS_CUDA_TRY(expr)                                  \
    do {                                                    \
        cudaError_t e__ = (expr);                           \
        if (e__ != cudaSuccess) return LCS_ERR_CUDA;        \
    } while (0)

#define LCS_LAUNCH_CHECK()                                  \
    do {                                                    \
        cudaError_t e__ = cudaGetLastError();               \
        if (e__ != cudaSuccess) return LCS_ERR_CUDA;        \
    } while (0)
