// radix_sort.cuh -- stable LSD radix sort of (key, uint32 value) pairs, 8-bit digits.
//
// Replaces the host CpuParallel::parallel_sort of LBVH::construct_tree (lbvh.cpp:983-993)
// and the 256-wide bitonic block sorts of the contact triplet reduction
// (reduce_helper.h:340-432, narrow_phase.cpp:1450-1591).  Each pass is three kernels:
//   upsweep : per-tile (2048 keys) digit histogram, digit-major  hist[d * tiles + tile]
//   scan    : one block per digit scans its row over tiles; row totals for the digit bases
//   scatter : stable in-tile ranks (rounds of 256 keys, warp match_any + per-warp digit
//             counts), written to digit_base[d] + row_prefix[d][tile] + rank
// The element count may live on the device (d_n), so a sort can sit inside a captured graph
// whose sizes are only known on the GPU; tiles beyond the count exit at once.
#pragma once
#include "lcs_common.cuh"

namespace lcs {
namespace rs {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ uint32_t count_of(const uint32_t* d_n, uint32_t n_host, uint32_t cap)
{
    uint32_t n = d_n ? *d_n : n_host;
    return n < cap ? n : cap;
}

template <typename K>
__global__ void __launch_bounds__(kThreads) upsweep(const K* __restrict__ keys, const uint32_t* d_n, uint32_t n_host,
                                                    uint32_t cap, int shift, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t cnt[256];
    const uint32_t n = count_of(d_n, n_host, cap);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        cnt[threadIdx.x] = 0;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kItems; ++r) {
            uint32_t idx = tile * kTile + r * kThreads + threadIdx.x;
            if (idx < n) atomicAdd(&cnt[(uint32_t)(keys[idx] >> shift) & 255u], 1u);
        }
        __syncthreads();
        hist[threadIdx.x * tiles + tile] = cnt[threadIdx.x];
        __syncthreads();
    }
}

// one block per digit: exclusive scan of hist[d][0..tiles) in place, row total to totals[d]
static __global__ void __launch_bounds__(kThreads) scan_rows(uint32_t* __restrict__ hist, uint32_t* __restrict__ totals,
                                                      const uint32_t* d_n, uint32_t n_host, uint32_t cap)
{
    __shared__ uint32_t warp_sums[kWarps];
    __shared__ uint32_t carry_s;
    const uint32_t n = count_of(d_n, n_host, cap);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t d = blockIdx.x;
    uint32_t* row = hist + (size_t)d * tiles;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (uint32_t base = 0; base < tiles; base += kThreads) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < tiles ? row[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane_id() >= (uint32_t)o) incl += t;
        }
        if (lane_id() == 31) warp_sums[threadIdx.x >> 5] = incl;
        __syncthreads();
        uint32_t wpre = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            uint32_t s = warp_sums[w];
            if (w < (int)(threadIdx.x >> 5)) wpre += s;
            total += s;
        }
        uint32_t carry = carry_s;
        if (i < tiles) row[i] = carry + wpre + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[d] = carry_s;
}

template <typename K>
__global__ void __launch_bounds__(kThreads) scatter(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                    K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                    const uint32_t* __restrict__ hist, const uint32_t* __restrict__ totals,
                                                    const uint32_t* d_n, uint32_t n_host, uint32_t cap, int shift)
{
    __shared__ uint32_t digit_base[256];
    __shared__ uint32_t warp_cnt[kWarps][256];
    __shared__ uint32_t running[256];
    __shared__ uint32_t wsum[kWarps];
    const uint32_t n = count_of(d_n, n_host, cap);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t t = threadIdx.x, w = t >> 5, lane = lane_id();
    // exclusive scan of the 256 digit totals -> digit bases
    {
        uint32_t v = totals[t], incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t s = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (uint32_t)o) incl += s;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        uint32_t pre = 0;
        for (uint32_t k = 0; k < w; ++k) pre += wsum[k];
        digit_base[t] = pre + incl - v;
    }
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        running[t] = 0;
#pragma unroll 1
        for (int r = 0; r < kItems; ++r) {
#pragma unroll
            for (int k = 0; k < kWarps; ++k) warp_cnt[k][t] = 0;
            __syncthreads();
            const uint32_t idx = tile * kTile + r * kThreads + t;
            const bool valid = idx < n;
            K key = 0;
            uint32_t val = 0, d = 0x100u;
            if (valid) {
                key = keys_in[idx];
                val = vals_in[idx];
                d = (uint32_t)(key >> shift) & 255u;
            }
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
            const uint32_t rank = __popc(peers & lt_mask);
            if (valid && rank == 0) warp_cnt[w][d] = __popc(peers);
            __syncthreads();
            {
                uint32_t acc = running[t];
#pragma unroll
                for (int k = 0; k < kWarps; ++k) {
                    uint32_t c = warp_cnt[k][t];
                    warp_cnt[k][t] = acc;
                    acc += c;
                }
                running[t] = acc;
            }
            __syncthreads();
            if (valid) {
                uint32_t pos = digit_base[d] + hist[(size_t)d * tiles + tile] + warp_cnt[w][d] + rank;
                keys_out[pos] = key;
                vals_out[pos] = val;
            }
            __syncthreads();
        }
    }
}

// bytes of histogram scratch for up to `cap` keys
inline size_t hist_words(uint32_t cap) { return (size_t)256 * ((cap + kTile - 1) / kTile) + 256; }

// Sorts (keys, vals) on bits [begin_bit, end_bit).  Ping-pongs with the alt buffers; returns
// true when the result ended in the alt buffers.  n on device (d_n) or host (d_n == NULL).
template <typename K>
inline bool sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, const uint32_t* d_n,
                       uint32_t n_host, uint32_t cap, int begin_bit, int end_bit, uint32_t* hist_scratch,
                       cudaStream_t s)
{
    const uint32_t max_tiles = (cap + kTile - 1) / kTile;
    if (max_tiles == 0) return false;
    uint32_t* totals = hist_scratch;
    uint32_t* hist = hist_scratch + 256;
    const int grid = (int)(max_tiles < 4u * kNumSMs ? max_tiles : 4u * kNumSMs);
    K* kin = keys;
    uint32_t* vin = vals;
    K* kout = keys_alt;
    uint32_t* vout = vals_alt;
    bool in_alt = false;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        upsweep<K><<<grid, kThreads, 0, s>>>(kin, d_n, n_host, cap, shift, hist);
        lcs_count_launch();
        scan_rows<<<256, kThreads, 0, s>>>(hist, totals, d_n, n_host, cap);
        lcs_count_launch();
        scatter<K><<<grid, kThreads, 0, s>>>(kin, vin, kout, vout, hist, totals, d_n, n_host, cap, shift);
        lcs_count_launch();
        K* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
        in_alt = !in_alt;
    }
    return in_alt;
}

}  // namespace rs
}  // namespace lcs
