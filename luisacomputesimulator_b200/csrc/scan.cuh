// scan.cuh -- exclusive prefix sum of uint32 with the element count on the device
// (block_intrinsic_scan_exclusive + the atomic block offsets of the reference,
// reduce_helper.h:142-185 and narrow_phase.cpp:1291-1315, but in a fixed order so results do
// not depend on block scheduling).  Three kernels: tile sums, scan of tile sums, tile scans.
#pragma once
#include "lcs_common.cuh"

namespace lcs {
namespace scan {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

inline size_t tmp_words(uint32_t cap) { return (size_t)(cap + kTile - 1) / kTile + 32; }

__device__ __forceinline__ uint32_t cnt(const uint32_t* d_n, uint32_t cap)
{
    uint32_t n = *d_n;
    return n < cap ? n : cap;
}

// block-wide inclusive scan of one value per thread; returns inclusive, writes block total
__device__ __forceinline__ uint32_t block_incl(uint32_t v, uint32_t& total)
{
    __shared__ uint32_t ws[kThreads / 32];
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane_id() >= (uint32_t)o) incl += t;
    }
    if (lane_id() == 31) ws[threadIdx.x >> 5] = incl;
    __syncthreads();
    uint32_t pre = 0;
    total = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        uint32_t s = ws[w];
        if (w < (int)(threadIdx.x >> 5)) pre += s;
        total += s;
    }
    __syncthreads();
    return pre + incl;
}

static __global__ void __launch_bounds__(kThreads) k_tile_sums(const uint32_t* __restrict__ in, const uint32_t* d_n, uint32_t cap,
                                                        uint32_t* __restrict__ sums)
{
    const uint32_t n = cnt(d_n, cap);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        uint32_t v = 0;
        const uint32_t base = tile * kTile + threadIdx.x * kItems;
#pragma unroll
        for (int k = 0; k < kItems; ++k)
            if (base + k < n) v += in[base + k];
        uint32_t total;
        block_incl(v, total);
        if (threadIdx.x == 0) sums[tile] = total;
    }
}

static __global__ void __launch_bounds__(kThreads) k_scan_sums(uint32_t* __restrict__ sums, const uint32_t* d_n, uint32_t cap)
{
    const uint32_t n = cnt(d_n, cap);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < tiles; base += kThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < tiles ? sums[i] : 0u;
        uint32_t total;
        const uint32_t incl = block_incl(v, total);
        const uint32_t c = carry;
        if (i < tiles) sums[i] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry = c + total;
        __syncthreads();
    }
}

static __global__ void __launch_bounds__(kThreads) k_tile_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                        const uint32_t* d_n, uint32_t cap,
                                                        const uint32_t* __restrict__ sums)
{
    const uint32_t n = cnt(d_n, cap);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        uint32_t v[kItems];
        uint32_t s = 0;
        const uint32_t base = tile * kTile + threadIdx.x * kItems;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            v[k] = base + k < n ? in[base + k] : 0u;
            s += v[k];
        }
        uint32_t total;
        uint32_t run = block_incl(s, total) - s + sums[tile];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (base + k < n) out[base + k] = run;
            run += v[k];
        }
    }
}

inline void exclusive_u32(const uint32_t* in, uint32_t* out, const uint32_t* d_n, uint32_t cap, uint32_t* tmp,
                          cudaStream_t s)
{
    const uint32_t max_tiles = (cap + kTile - 1) / kTile;
    if (!max_tiles) return;
    const int grid = (int)(max_tiles < 4u * kNumSMs ? max_tiles : 4u * kNumSMs);
    k_tile_sums<<<grid, kThreads, 0, s>>>(in, d_n, cap, tmp);
    lcs_count_launch();
    k_scan_sums<<<1, kThreads, 0, s>>>(tmp, d_n, cap);
    lcs_count_launch();
    k_tile_scan<<<grid, kThreads, 0, s>>>(in, out, d_n, cap, tmp);
    lcs_count_launch();
}

}  // namespace scan
}  // namespace lcs
