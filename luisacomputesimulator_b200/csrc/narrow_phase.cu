// narrow_phase.cu -- VF/EE additive CCD, VF/EE barrier DCD, contact gradient / diagonal
// assembly, contact energy, and the contact off-diagonal blocks as BSR.
//
// Reference: Solver/CollisionDetector/narrow_phase.cpp (citations per kernel).  Candidate
// lists are processed by grid-stride loops over min(*d_count, capacity) pairs, so the count
// can stay on the device (no host read-back between broad and narrow phase).
#include <cuda_runtime.h>

#include <new>

#include "lcs_common.cuh"
#include "lcs_geom.cuh"
#include "lbvh_common.cuh"
#include "lcs_internal.h"
#include "radix_sort.cuh"
#include "scan.cuh"
#include "abd.cuh"

using namespace lcs;

namespace {

// float atomic min valid for either sign
__device__ __forceinline__ void atomic_min_float(float* addr, float v)
{
    if (v >= 0.0f)
        atomicMin(reinterpret_cast<int*>(addr), __float_as_int(v));
    else
        atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}

__device__ __forceinline__ float block_min(float v)
{
    __shared__ float red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmn(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    if (lane_id() == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmn(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    }
    return v;
}

// fn_narrow_phase_vf_ccd_query (EE = false, narrow_phase.cpp:293-436) and
// fn_narrow_phase_ee_ccd_query (EE = true, narrow_phase.cpp:438-593)
// F64: the precision form's all-FP64 iteration (LCS_CCD_FP64), a separate instantiation so the
// FP32 kernel keeps its register budget
template <bool EE, bool F64>
__global__ void __launch_bounds__(256) k_ccd(const uint2* __restrict__ pairs, const uint32_t* d_count, uint32_t cap,
                                             const float4* __restrict__ x0, const float4* __restrict__ x1,
                                             const uint32_t* __restrict__ elems, const uint32_t* __restrict__ body,
                                             const float* __restrict__ offset, float* d_toi,
                                             float* __restrict__ toi_per_pair, int flags,
                                             const uint32_t* __restrict__ vscene)
{
    const bool fp64_final = (flags & LCS_CCD_FP64_FINAL) != 0;
    const uint32_t n = pair_count(d_count, cap);
    float local = 1.0f;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint2 pr = __ldg(&pairs[p]);
        float toi = 1.25f;
        v3 a[4], b[4];
        uint32_t v[4];
        bool skip;
        if (EE) {
            uint2 l = __ldg(reinterpret_cast<const uint2*>(elems) + pr.x);
            uint2 r = __ldg(reinterpret_cast<const uint2*>(elems) + pr.y);
            v[0] = l.x; v[1] = l.y; v[2] = r.x; v[3] = r.y;
            const uint32_t bl = __ldg(&body[l.x]);
            skip = l.x == r.x || l.x == r.y || l.y == r.x || l.y == r.y || (bl != kInvalid && bl == __ldg(&body[r.x]));
        } else {
            uint4 f = __ldg(reinterpret_cast<const uint4*>(elems) + pr.y);
            v[0] = pr.x; v[1] = f.x; v[2] = f.y; v[3] = f.z;
            const uint32_t bv = __ldg(&body[pr.x]);
            skip = pr.x == f.x || pr.x == f.y || pr.x == f.z || (bv != kInvalid && bv == __ldg(&body[f.x]));
        }
        if (!skip) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                a[k] = ld3(x0, v[k]);
                b[k] = ld3(x1, v[k]);
            }
            const float th = __ldg(&offset[v[0]]) + __ldg(&offset[EE ? v[2] : v[1]]);
            toi = F64 ? __double2float_rz(accd_ccd_f64<EE>(a, b, th)) : accd_ccd<EE>(a, b, th, fp64_final);
        }
        if (toi_per_pair) toi_per_pair[p] = toi;
        if (vscene) {  // batched scenes: the bound of the pair's own scene
            const float g = toi / 1.25f;
            if (g < 1.0f) atomic_min_float(d_toi + __ldg(&vscene[EE ? v[0] : pr.x]), g);
        } else {
            local = fmn(local, toi / 1.25f);
        }
    }
    if (vscene) return;
    const float m = block_min(local);
    if (threadIdx.x == 0 && m < 1.0f) atomic_min_float(d_toi, m);
}

__device__ __forceinline__ void write_pair(lcs_pair* out, uint32_t s, uint32_t i0, uint32_t i1, uint32_t i2,
                                           uint32_t i3, v3 n, float k1, float k2, float stiff, float b0, float b1)
{
    uint4* o = reinterpret_cast<uint4*>(out + s);
    o[0] = make_uint4(i0, i1, i2, i3);
    reinterpret_cast<float4*>(o)[1] = make_float4(n.x, n.y, n.z, stiff);
    reinterpret_cast<float4*>(o)[2] = make_float4(k1, k2, b0, b1);
}

// The candidate test of lcs_candidates_filter: a swept-box candidate whose static boxes overlap at x (the
// query box +- thickness + d_hat of its first vertex, the leaf box +- thickness of its element's first
// vertex, strict).  With FILTER the DCD kernels below take the previous iteration's CCD list and count the
// candidates passing it into d_cand_count themselves -- the DCD list lcs_candidates_filter would write is the
// same set, so the pairs and counts are those of filter + DCD.
template <bool EE>
__device__ __forceinline__ bool static_candidate(uint2 pr, const float4* __restrict__ x, const uint32_t* __restrict__ elems,
                                                 const float* __restrict__ dhat, const float* __restrict__ thickness)
{
    v3 mn, mx;
    uint32_t v0;
    if (EE) {
        const uint2 ed = __ldg(reinterpret_cast<const uint2*>(elems) + pr.x);
        const v3 s0 = ld3(x, ed.x), s1 = ld3(x, ed.y);
        mn = min3(min3(s0, s1), min3(s0, s1));
        mx = max3(max3(s0, s1), max3(s0, s1));
        v0 = ed.x;
    } else {
        const v3 qa = ld3(x, pr.x);
        mn = min3(qa, qa);
        mx = max3(qa, qa);
        v0 = pr.x;
    }
    const float r = __ldg(&thickness[v0]) + __ldg(&dhat[v0]);
    const float q[6] = {mn.x - r, mn.y - r, mn.z - r, mx.x + r, mx.y + r, mx.z + r};
    v3 lm, lx;
    leaf_box(EE ? LCS_TREE_EDGE : LCS_TREE_FACE, pr.y, thickness, x, x, elems, lm, lx);
    return overlap(make_float4(lm.x, lm.y, lm.z, 0.f), make_float4(lx.x, lx.y, lx.z, 0.f), q);
}

// fn_narrow_phase_vf_dcd_query (barrier energy), narrow_phase.cpp:771-933
template <bool FILTER>
__global__ void __launch_bounds__(256) k_dcd_vf(const uint2* __restrict__ pairs, const uint32_t* d_count, uint32_t cap,
                                                const float4* __restrict__ x, const uint4* __restrict__ faces,
                                                const uint32_t* __restrict__ body, const float* __restrict__ vert_area,
                                                const float* __restrict__ face_area, const float* __restrict__ dhat,
                                                const float* __restrict__ offset, float kappa, lcs_pair* out,
                                                uint32_t out_cap, uint32_t* d_out_count, uint32_t* d_cand_count)
{
    const uint32_t n = pair_count(d_count, cap);
    const uint32_t n_round = (n + 31u) & ~31u;  // whole warps iterate together for the append
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_round; p += gridDim.x * blockDim.x) {
        bool emit = false;
        uint32_t vid = 0, fid = 0;
        uint4 f = make_uint4(0, 0, 0, 0);
        v3 nrm = mk3(0, 0, 0);
        float k1 = 0, k2 = 0, stiff = 0, c0 = 0, c1 = 0;
        bool cand = false;
        if (p < n) {
            const uint2 pr = __ldg(&pairs[p]);
            cand = !FILTER || static_candidate<false>(pr, x, reinterpret_cast<const uint32_t*>(faces), dhat, offset);
            vid = pr.x;
            fid = pr.y;
            f = __ldg(&faces[fid]);
            const uint32_t bv = __ldg(&body[vid]);
            const bool skip = !cand || vid == f.x || vid == f.y || vid == f.z ||
                              (bv != kInvalid && bv == __ldg(&body[f.x]));
            if (!skip) {
                const v3 pp = ld3(x, vid), t0 = ld3(x, f.x), t1 = ld3(x, f.y), t2 = ld3(x, f.z);
                float c[3];
                Gf::pt_coeff(tovf(pp), tovf(t0), tovf(t1), tovf(t2), c);
                const v3 xv = (c[0] * (pp - t0) + c[1] * (pp - t1)) + c[2] * (pp - t2);
                const float d2 = dot3(xv, xv);
                const float dh = (__ldg(&dhat[vid]) + __ldg(&dhat[f.x])) * 0.5f;
                const float th = __ldg(&offset[vid]) + __ldg(&offset[f.x]);
                const float lim = th + dh;
                if (d2 < lim * lim) {
                    const float d = sqrtf(d2);
                    nrm = mk3(xv.x / d, xv.y / d, xv.z / d);
                    const float area = 0.5f * (__ldg(&vert_area[vid]) + __ldg(&face_area[fid]));
                    k1 = -area * kappa * barrier_d1(d - th, dh);
                    k2 = area * kappa * barrier_d2(d - th, dh);
                    stiff = area * kappa;
                    c0 = c[0];
                    c1 = c[1];
                    emit = true;
                }
            }
        }
        if (FILTER) warp_append(d_cand_count, cand);
        const uint32_t s = warp_append(d_out_count, emit);
        if (emit && s < out_cap) write_pair(out, s, vid, f.x, f.y | 0x80000000u, f.z, nrm, k1, k2, stiff, c0, c1);
    }
}

// fn_narrow_phase_ee_dcd_query (barrier energy), narrow_phase.cpp:935-1098
template <bool FILTER>
__global__ void __launch_bounds__(256) k_dcd_ee(const uint2* __restrict__ pairs, const uint32_t* d_count, uint32_t cap,
                                                const float4* __restrict__ x, const uint2* __restrict__ edges,
                                                const uint32_t* __restrict__ body, const float* __restrict__ edge_area,
                                                const float* __restrict__ dhat, const float* __restrict__ offset,
                                                float kappa, lcs_pair* out, uint32_t out_cap, uint32_t* d_out_count,
                                                uint32_t* d_cand_count)
{
    const uint32_t n = pair_count(d_count, cap);
    const uint32_t n_round = (n + 31u) & ~31u;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_round; p += gridDim.x * blockDim.x) {
        bool emit = false;
        uint2 l = make_uint2(0, 0), r = make_uint2(0, 0);
        v3 nrm = mk3(0, 0, 0);
        float k1 = 0, k2 = 0, stiff = 0, c0 = 0, c2 = 0;
        bool cand = false;
        if (p < n) {
            const uint2 pr = __ldg(&pairs[p]);
            cand = !FILTER || static_candidate<true>(pr, x, reinterpret_cast<const uint32_t*>(edges), dhat, offset);
            l = __ldg(&edges[pr.x]);
            r = __ldg(&edges[pr.y]);
            const uint32_t bl = __ldg(&body[l.x]);
            const bool skip = !cand || l.x == r.x || l.x == r.y || l.y == r.x || l.y == r.y ||
                              (bl != kInvalid && bl == __ldg(&body[r.x]));
            if (!skip) {
                const v3 ea0 = ld3(x, l.x), ea1 = ld3(x, l.y), eb0 = ld3(x, r.x), eb1 = ld3(x, r.y);
                float c[4];
                Gf::ee_coeff(tovf(ea0), tovf(ea1), tovf(eb0), tovf(eb1), c);
                const v3 xa = c[0] * ea0 + c[1] * ea1;
                const v3 xb = c[2] * eb0 + c[3] * eb1;
                const v3 xv = xa - xb;
                const float d2 = dot3(xv, xv);
                const float dh = (__ldg(&dhat[l.x]) + __ldg(&dhat[r.x])) * 0.5f;
                const float th = __ldg(&offset[l.x]) + __ldg(&offset[r.x]);
                const float lim = th + dh;
                if (d2 < lim * lim) {
                    const float d = sqrtf(d2);
                    nrm = mk3(xv.x / d, xv.y / d, xv.z / d);
                    const float area = 0.5f * (__ldg(&edge_area[pr.x]) + __ldg(&edge_area[pr.y]));
                    k1 = -area * kappa * barrier_d1(d - th, dh);
                    k2 = area * kappa * barrier_d2(d - th, dh);
                    stiff = area * kappa;
                    c0 = c[0];
                    c2 = c[2];
                    emit = true;
                }
            }
        }
        if (FILTER) warp_append(d_cand_count, cand);
        const uint32_t s = warp_append(d_out_count, emit);
        if (emit && s < out_cap) write_pair(out, s, l.x, l.y, r.x, r.y | 0x80000000u, nrm, k1, k2, stiff, c0, c2);
    }
}

// fn_perPair_assemble_gradient_hessian, narrow_phase.cpp:2550-2676: b += k1 w n and D += k2 w^2 n n^T for
// every generalised DOF of the pair (soft vertices, or a rigid side's four DOF slots)
template <bool ABD>
__global__ void __launch_bounds__(256) k_grad_diag(const lcs_pair* __restrict__ pairs, const uint32_t* d_count,
                                                   uint32_t cap, float* b, float* diag, AbdView abd)
{
    const uint32_t n = pair_count(d_count, cap);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const PairView P = load_pair(pairs, k);
        if (!P.type) continue;
        const float nn[3] = {P.n.x, P.n.y, P.n.z};
        uint32_t dof[8];
        float gw[8];
        int nd = 4;
        if (ABD) {
            nd = pair_dofs(P, abd, dof, gw);
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                dof[i] = P.v[i];
                gw[i] = P.w[i];
            }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if (i >= nd) break;
            const float g = P.k1 * gw[i];
            float* bv = b + 4 * (size_t)dof[i];
            atomicAdd(bv + 0, g * P.n.x);
            atomicAdd(bv + 1, g * P.n.y);
            atomicAdd(bv + 2, g * P.n.z);
            const float h = P.k2 * gw[i] * gw[i];
            float* dv = diag + 12 * (size_t)dof[i];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r) atomicAdd(dv + 4 * c + r, h * (nn[r] * nn[c]));
        }
    }
}

// fn_compute_repulsion_energy (barrier), narrow_phase.cpp:2968-3044; FP64 accumulation
__global__ void __launch_bounds__(256) k_energy(const lcs_pair* __restrict__ pairs, const uint32_t* d_count,
                                                uint32_t cap, const float4* __restrict__ x,
                                                const float* __restrict__ dhat, const float* __restrict__ offset,
                                                double* d_energy)
{
    __shared__ double red[8];
    const uint32_t n = pair_count(d_count, cap);
    double acc = 0.0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const PairView P = load_pair(pairs, k);
        if (!P.type) continue;
        const v3 diff = ((P.w[0] * ld3(x, P.v[0]) + P.w[1] * ld3(x, P.v[1])) + P.w[2] * ld3(x, P.v[2])) +
                        P.w[3] * ld3(x, P.v[3]);
        const float d = sqrtf(dot3(diff, diff));
        const float dh = 0.5f * (__ldg(&dhat[P.v[0]]) + __ldg(&dhat[P.v[2]]));
        const float th = __ldg(&offset[P.v[0]]) + __ldg(&offset[P.v[2]]);
        if (d < th + dh) acc += (double)(P.stiff * barrier_e(d - th, dh));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane_id() == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += red[w];
        if (s != 0.0) atomicAdd(d_energy, s);
    }
}

// ---------------------------------------------------------------- off-diagonal blocks (BSR)
// key = row << bits | col; value = pair * 16 + i * 4 + j: 12 directed (i, j) per pair.  With affine
// bodies the pair's generalised DOFs (up to 8) give up to 56 directed pairs, value = pair * 64 + i * 8 + j,
// unused entries sorting last like non-contact ones.
template <bool ABD>
__global__ void k_trip_keys(const lcs_pair* __restrict__ pairs, const uint32_t* d_count, uint32_t cap, int bits,
                            uint32_t n_rows, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                            uint32_t* d_ntrip, AbdView abd)
{
    constexpr uint32_t T = ABD ? 56u : 12u;
    const uint32_t n = pair_count(d_count, cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_ntrip = T * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const PairView P = load_pair(pairs, k);
        if (!ABD) {
            int t = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (i != j) {
                        const uint64_t row = P.type ? P.v[i] : n_rows;  // non-contact entries sort last, dropped
                        keys[12 * (size_t)k + t] = (row << bits) | (uint64_t)P.v[j];
                        vals[12 * (size_t)k + t] = 16u * k + 4u * i + j;
                        ++t;
                    }
        } else {
            uint32_t dof[8];
            float gw[8];
            const int nd = P.type ? pair_dofs(P, abd, dof, gw) : 0;
            uint32_t t = 0;
            for (int i = 0; i < nd; ++i)
                for (int j = 0; j < nd; ++j)
                    if (i != j) {
                        keys[T * (size_t)k + t] = ((uint64_t)dof[i] << bits) | (uint64_t)dof[j];
                        vals[T * (size_t)k + t] = 64u * k + 8u * i + j;
                        ++t;
                    }
            for (; t < T; ++t) {
                keys[T * (size_t)k + t] = (uint64_t)n_rows << bits;
                vals[T * (size_t)k + t] = 64u * k;
            }
        }
    }
}

__global__ void k_heads(const uint64_t* __restrict__ keys, const uint32_t* d_n, uint32_t cap, int bits,
                        uint32_t n_rows, uint32_t* __restrict__ flags)
{
    const uint32_t n = pair_count(d_n, cap);
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint64_t k = keys[s];
        flags[s] = ((s == 0 || k != keys[s - 1]) && (uint32_t)(k >> bits) < n_rows) ? 1u : 0u;
    }
}

// segmented sum in sorted (key, pair, i, j) order -- the oracle's order, so values match bitwise
// (fn_assemble_triplet_sorted, narrow_phase.cpp:1760-1880)
template <bool ABD>
__global__ void k_segments(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                           const uint32_t* __restrict__ flags, const uint32_t* __restrict__ excl,
                           const uint32_t* d_n, uint32_t cap, int bits, uint32_t n_rows,
                           const lcs_pair* __restrict__ pairs, uint32_t* __restrict__ col, uint32_t* __restrict__ brow,
                           float* __restrict__ val, uint32_t* d_nnzb, AbdView abd)
{
    const uint32_t n = pair_count(d_n, cap);
    const uint64_t cmask = (1ull << bits) - 1ull;
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_nnzb = n ? excl[n - 1] + flags[n - 1] : 0u;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        if (!flags[s]) continue;
        const uint64_t key = keys[s];
        const uint32_t b = excl[s];
        col[b] = (uint32_t)(key & cmask);
        brow[b] = (uint32_t)(key >> bits);
        float acc[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) acc[q] = 0.0f;
        for (uint32_t t = s; t < n && keys[t] == key; ++t) {
            const uint32_t v = vals[t];
            float sw;
            PairView P;
            if (ABD) {
                P = load_pair(pairs, v >> 6);
                uint32_t dof[8];
                float gw[8];
                pair_dofs(P, abd, dof, gw);
                sw = gw[(v >> 3) & 7u] * gw[v & 7u];
            } else {
                P = load_pair(pairs, v >> 4);
                sw = P.w[(v >> 2) & 3u] * P.w[v & 3u];
            }
            const float nn[3] = {P.n.x, P.n.y, P.n.z};
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r) acc[3 * c + r] += sw * (P.k2 * (nn[r] * nn[c]));
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) val[9 * (size_t)b + q] = acc[q];
    }
}

// The (row, column, triplet) order of the contact triplets without a global radix sort (pairs without affine
// bodies): the 12 directed vertex pairs of every contact pair are bucketed by row (a count, a scan and a
// scatter with per-row cursors), and each entry finds its place in its row's bucket by counting the entries
// that precede it in (column, triplet index) order -- the order the stable radix sort gives.  Rows hold at
// most a few hundred entries.  k_heads, k_segments and k_row_ptr then run on the result as after the sort.
__global__ void k_row_count(const lcs_pair* __restrict__ pairs, const uint32_t* d_count, uint32_t cap,
                            uint32_t* __restrict__ rcnt)
{
    const uint32_t n = pair_count(d_count, cap);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const PairView P = load_pair(pairs, k);
        if (!P.type) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) atomicAdd(&rcnt[P.v[i]], 3u);
    }
}

__global__ void k_row_scatter(const lcs_pair* __restrict__ pairs, const uint32_t* d_count, uint32_t cap, int bits,
                              const uint32_t* __restrict__ rstart, uint32_t* __restrict__ rcur,
                              uint64_t* __restrict__ tkeys, uint32_t* __restrict__ tvals)
{
    const uint32_t n = pair_count(d_count, cap);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const PairView P = load_pair(pairs, k);
        if (!P.type) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t base = rstart[P.v[i]] + atomicAdd(&rcur[P.v[i]], 3u);
            uint32_t t = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (i != j) {
                    tkeys[base + t] = ((uint64_t)P.v[i] << bits) | (uint64_t)P.v[j];
                    tvals[base + t] = 16u * k + 4u * i + j;
                    ++t;
                }
        }
    }
}

__global__ void k_row_rank(uint32_t n_rows, const uint32_t* __restrict__ rstart, int bits,
                           const uint64_t* __restrict__ tkeys, const uint32_t* __restrict__ tvals,
                           uint64_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t* d_n)
{
    const uint32_t n = rstart[n_rows];
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_n = n;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint64_t k = tkeys[e];
        const uint32_t v = tvals[e];
        const uint32_t r = (uint32_t)(k >> bits);
        const uint32_t lo = rstart[r], hi = rstart[r + 1];
        uint32_t rank = 0;
        for (uint32_t q = lo; q < hi; ++q) {
            const uint64_t kq = tkeys[q];
            rank += (kq < k || (kq == k && tvals[q] < v)) ? 1u : 0u;
        }
        keys[lo + rank] = k;
        vals[lo + rank] = v;
    }
}

// row_ptr[r] = first block whose row >= r (binary search over the sorted block rows)
__global__ void k_row_ptr(const uint32_t* __restrict__ brow, const uint32_t* d_nnzb, uint32_t n_rows,
                          uint32_t* __restrict__ row_ptr)
{
    const uint32_t nb = *d_nnzb;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= n_rows; r += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nb;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (brow[mid] < r) lo = mid + 1; else hi = mid;
        }
        row_ptr[r] = lo;
    }
}

}  // namespace

struct lcs_assembler {
    uint32_t n_rows = 0, pair_cap = 0, trip_cap = 0;
    bool abd = false;  // sized for pairs with affine-body sides (56 directed DOF pairs each)
    int bits = 1;
    uint64_t *keys = nullptr, *keys_alt = nullptr;
    uint32_t *vals = nullptr, *vals_alt = nullptr, *hist = nullptr;
    uint32_t *flags = nullptr, *excl = nullptr, *scan_tmp = nullptr;
    uint32_t *d_ntrip = nullptr, *d_nnzb = nullptr;
    uint32_t *row_ptr = nullptr, *col = nullptr, *brow = nullptr;
    float* val = nullptr;
    // row bucketing (pairs without affine bodies): per-row counts / starts / cursors, n_rows + 1 each
    uint32_t *rcnt = nullptr, *rstart = nullptr, *rcur = nullptr, *d_rows1 = nullptr;
    uint32_t* rscan_tmp = nullptr;
};

namespace {
int assembler_create(uint32_t n_rows, uint32_t pair_capacity, bool abd, lcs_assembler** out)
{
    if (!out || n_rows == 0) return lcs_fail(LCS_ERR_INVALID, "lcs_assembler_create: bad argument");
    lcs_assembler* a = new (std::nothrow) lcs_assembler();
    if (!a) return lcs_fail(LCS_ERR_INVALID, "lcs_assembler_create: out of host memory");
    a->n_rows = n_rows;
    a->abd = abd;
    a->pair_cap = pair_capacity ? pair_capacity : 1;
    a->trip_cap = (abd ? 56u : 12u) * a->pair_cap;
    int bits = 1;
    while ((1ull << bits) <= (uint64_t)n_rows) ++bits;  // rows up to n_rows (the drop marker) fit
    a->bits = bits;
    const size_t T = a->trip_cap;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 4); };
    A((void**)&a->keys, 8 * T);
    A((void**)&a->keys_alt, 8 * T);
    A((void**)&a->vals, 4 * T);
    A((void**)&a->vals_alt, 4 * T);
    A((void**)&a->hist, 4 * rs::hist_words(a->trip_cap));
    A((void**)&a->flags, 4 * T);
    A((void**)&a->excl, 4 * T);
    A((void**)&a->scan_tmp, 4 * scan::tmp_words(a->trip_cap));
    A((void**)&a->d_ntrip, 4);
    A((void**)&a->d_nnzb, 4);
    A((void**)&a->row_ptr, 4 * ((size_t)n_rows + 1));
    A((void**)&a->col, 4 * T);
    A((void**)&a->brow, 4 * T);
    A((void**)&a->val, 36 * T);
    const size_t R1 = (size_t)n_rows + 1;
    A((void**)&a->rcnt, 4 * R1);
    A((void**)&a->rstart, 4 * R1);
    A((void**)&a->rcur, 4 * R1);
    A((void**)&a->d_rows1, 4);
    A((void**)&a->rscan_tmp, 4 * scan::tmp_words((uint32_t)R1));
    if (e == cudaSuccess) {
        const uint32_t r1 = (uint32_t)R1;
        e = cudaMemcpy(a->d_rows1, &r1, 4, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(a->row_ptr, 0, 4 * ((size_t)n_rows + 1));
    if (e == cudaSuccess) e = cudaMemset(a->d_nnzb, 0, 4);
    if (e != cudaSuccess) {
        lcs_assembler_destroy(a);
        return lcs_fail(LCS_ERR_CUDA, "lcs_assembler_create: cudaMalloc failed");
    }
    *out = a;
    return LCS_OK;
}
}  // namespace

extern "C" int lcs_assembler_create(uint32_t n_rows, uint32_t pair_capacity, lcs_assembler** out)
{
    return assembler_create(n_rows, pair_capacity, false, out);
}

extern "C" int lcs_assembler_create_abd(uint32_t n_rows, uint32_t pair_capacity, lcs_assembler** out)
{
    return assembler_create(n_rows, pair_capacity, true, out);
}

extern "C" int lcs_assembler_destroy(lcs_assembler* a)
{
    if (!a) return LCS_OK;
    void* ptrs[] = {a->keys, a->keys_alt, a->vals, a->vals_alt, a->hist, a->flags, a->excl, a->scan_tmp,
                    a->d_ntrip, a->d_nnzb, a->row_ptr, a->col, a->brow, a->val, a->rcnt, a->rstart, a->rcur,
                    a->d_rows1, a->rscan_tmp};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete a;
    return LCS_OK;
}

namespace {
AbdView abd_view(const lcs_abd_view* v)
{
    return v ? AbdView{v->body, reinterpret_cast<const float4*>(v->model_x), v->body_dof} : AbdView{nullptr, nullptr, nullptr};
}

int offdiag_bsr(lcs_assembler* a, const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity,
                const lcs_abd_view* abdv, lcs_stream stream)
{
    if (!a || !pairs || !d_count) return lcs_fail(LCS_ERR_INVALID, "lcs_contact_offdiag_bsr: bad argument");
    if (capacity > a->pair_cap) return lcs_fail(LCS_ERR_CAPACITY, "lcs_contact_offdiag_bsr: capacity above the assembler's");
    const bool abd = abdv != nullptr;
    if (abd && (!a->abd || !abdv->body || !abdv->model_x || !abdv->body_dof))
        return lcs_fail(LCS_ERR_INVALID, "lcs_contact_offdiag_bsr_abd: assembler not created for affine bodies, or view incomplete");
    const AbdView av = abd_view(abdv);
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t tcap = (abd ? 56u : 12u) * capacity;
    const uint64_t* keys;
    const uint32_t* vals;
    if (!abd) {  // row bucketing: count, scan, scatter, rank within the row
        const uint32_t R1 = a->n_rows + 1;
        LCS_CUDA_TRY(cudaMemsetAsync(a->rcnt, 0, 4 * (size_t)R1, s));
        LCS_CUDA_TRY(cudaMemsetAsync(a->rcur, 0, 4 * (size_t)R1, s));
        if (capacity) {
            k_row_count<<<grid_for(capacity, 256), 256, 0, s>>>(pairs, d_count, capacity, a->rcnt);
            lcs_count_launch();
        }
        scan::exclusive_u32(a->rcnt, a->rstart, a->d_rows1, R1, a->rscan_tmp, s);
        if (capacity) {
            k_row_scatter<<<grid_for(capacity, 256), 256, 0, s>>>(pairs, d_count, capacity, a->bits, a->rstart, a->rcur,
                                                                   a->keys_alt, a->vals_alt);
            lcs_count_launch();
        }
        k_row_rank<<<grid_for(tcap, 256), 256, 0, s>>>(a->n_rows, a->rstart, a->bits, a->keys_alt, a->vals_alt,
                                                       a->keys, a->vals, a->d_ntrip);
        lcs_count_launch();
        keys = a->keys;
        vals = a->vals;
    } else {
        k_trip_keys<true><<<grid_for(capacity, 256), 256, 0, s>>>(pairs, d_count, capacity, a->bits, a->n_rows,
                                                                  a->keys, a->vals, a->d_ntrip, av);
        lcs_count_launch();
        const bool alt = rs::sort_pairs<uint64_t>(a->keys, a->vals, a->keys_alt, a->vals_alt, a->d_ntrip, 0, tcap, 0,
                                                  2 * a->bits, a->hist, s);
        keys = alt ? a->keys_alt : a->keys;
        vals = alt ? a->vals_alt : a->vals;
    }
    const int g = grid_for(tcap, 256);
    k_heads<<<g, 256, 0, s>>>(keys, a->d_ntrip, tcap, a->bits, a->n_rows, a->flags);
    lcs_count_launch();
    scan::exclusive_u32(a->flags, a->excl, a->d_ntrip, tcap, a->scan_tmp, s);
    if (abd)
        k_segments<true><<<g, 256, 0, s>>>(keys, vals, a->flags, a->excl, a->d_ntrip, tcap, a->bits, a->n_rows, pairs,
                                           a->col, a->brow, a->val, a->d_nnzb, av);
    else
        k_segments<false><<<g, 256, 0, s>>>(keys, vals, a->flags, a->excl, a->d_ntrip, tcap, a->bits, a->n_rows,
                                            pairs, a->col, a->brow, a->val, a->d_nnzb, av);
    lcs_count_launch();
    k_row_ptr<<<grid_for(a->n_rows + 1, 256), 256, 0, s>>>(a->brow, a->d_nnzb, a->n_rows, a->row_ptr);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

int grad_diag(const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity, float* b, float* diag,
              const lcs_abd_view* abdv, lcs_stream stream)
{
    if (!d_count || !b || !diag || (capacity && !pairs)) return lcs_fail(LCS_ERR_INVALID, "lcs_contact_grad_diag: bad argument");
    if (abdv && (!abdv->body || !abdv->model_x || !abdv->body_dof))
        return lcs_fail(LCS_ERR_INVALID, "lcs_contact_grad_diag_abd: incomplete view");
    if (capacity == 0) return LCS_OK;
    if (abdv)
        k_grad_diag<true><<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(pairs, d_count, capacity, b, diag,
                                                                                     abd_view(abdv));
    else
        k_grad_diag<false><<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(pairs, d_count, capacity, b,
                                                                                      diag, abd_view(nullptr));
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}
}  // namespace

extern "C" int lcs_contact_offdiag_bsr(lcs_assembler* a, const lcs_pair* pairs, const uint32_t* d_count,
                                       uint32_t capacity, lcs_stream stream)
{
    return offdiag_bsr(a, pairs, d_count, capacity, nullptr, stream);
}

extern "C" int lcs_contact_offdiag_bsr_abd(lcs_assembler* a, const lcs_pair* pairs, const uint32_t* d_count,
                                           uint32_t capacity, const lcs_abd_view* abd, lcs_stream stream)
{
    if (!abd) return lcs_fail(LCS_ERR_INVALID, "lcs_contact_offdiag_bsr_abd: null view");
    return offdiag_bsr(a, pairs, d_count, capacity, abd, stream);
}

extern "C" int lcs_assembler_bsr(const lcs_assembler* a, lcs_bsr* out, const uint32_t** d_nnzb)
{
    if (!a || !out) return lcs_fail(LCS_ERR_INVALID, "lcs_assembler_bsr: bad argument");
    out->n_rows = a->n_rows;
    out->row_ptr = a->row_ptr;
    out->col = a->col;
    out->val = a->val;
    if (d_nnzb) *d_nnzb = a->d_nnzb;
    return LCS_OK;
}

extern "C" int lcs_assembler_export(const lcs_assembler* a, uint32_t* row_ptr, uint32_t* col, float* val,
                                    uint32_t max_blocks, uint32_t* nnzb, lcs_stream stream)
{
    if (!a || !nnzb) return lcs_fail(LCS_ERR_INVALID, "lcs_assembler_export: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    LCS_CUDA_TRY(cudaMemcpyAsync(nnzb, a->d_nnzb, 4, cudaMemcpyDeviceToHost, s));
    LCS_CUDA_TRY(cudaStreamSynchronize(s));
    const uint32_t nb = *nnzb < max_blocks ? *nnzb : max_blocks;
    if (row_ptr) LCS_CUDA_TRY(cudaMemcpyAsync(row_ptr, a->row_ptr, 4 * ((size_t)a->n_rows + 1), cudaMemcpyDeviceToDevice, s));
    if (col && nb) LCS_CUDA_TRY(cudaMemcpyAsync(col, a->col, 4 * (size_t)nb, cudaMemcpyDeviceToDevice, s));
    if (val && nb) LCS_CUDA_TRY(cudaMemcpyAsync(val, a->val, 36 * (size_t)nb, cudaMemcpyDeviceToDevice, s));
    LCS_CUDA_TRY(cudaStreamSynchronize(s));
    return *nnzb <= max_blocks ? LCS_OK : lcs_fail(LCS_ERR_CAPACITY, "lcs_assembler_export: more blocks than max_blocks");
}

extern "C" int lcs_ccd_vf(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x0,
                          const float* x1, const uint32_t* faces, const uint32_t* body, const float* offset,
                          float* d_toi, float* toi_per_pair, int flags, lcs_stream stream)
{
    if (!d_count || !x0 || !x1 || !faces || !body || !offset || !d_toi || (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_ccd_vf: bad argument");
    if (capacity == 0) return LCS_OK;
    auto kern = (flags & LCS_CCD_FP64) ? k_ccd<false, true> : k_ccd<false, false>;
    kern<<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(pairs), d_count, capacity, reinterpret_cast<const float4*>(x0),
        reinterpret_cast<const float4*>(x1), faces, body, offset, d_toi, toi_per_pair, flags, nullptr);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_ccd_ee(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x0,
                          const float* x1, const uint32_t* edges, const uint32_t* body, const float* offset,
                          float* d_toi, float* toi_per_pair, int flags, lcs_stream stream)
{
    if (!d_count || !x0 || !x1 || !edges || !body || !offset || !d_toi || (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_ccd_ee: bad argument");
    if (capacity == 0) return LCS_OK;
    auto kern = (flags & LCS_CCD_FP64) ? k_ccd<true, true> : k_ccd<true, false>;
    kern<<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(pairs), d_count, capacity, reinterpret_cast<const float4*>(x0),
        reinterpret_cast<const float4*>(x1), edges, body, offset, d_toi, toi_per_pair, flags, nullptr);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_ccd_batch(int is_ee, const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity,
                             const float* x0, const float* x1, const uint32_t* elems, const uint32_t* body,
                             const float* offset, const uint32_t* vert_scene, float* d_toi_per_scene,
                             float* toi_per_pair, int flags, lcs_stream stream)
{
    if (!d_count || !x0 || !x1 || !elems || !body || !offset || !vert_scene || !d_toi_per_scene || (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_ccd_batch: bad argument");
    if (capacity == 0) return LCS_OK;
    const bool f64 = (flags & LCS_CCD_FP64) != 0;
    auto kern = is_ee ? (f64 ? k_ccd<true, true> : k_ccd<true, false>) : (f64 ? k_ccd<false, true> : k_ccd<false, false>);
    kern<<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(pairs), d_count, capacity, reinterpret_cast<const float4*>(x0),
        reinterpret_cast<const float4*>(x1), elems, body, offset, d_toi_per_scene, toi_per_pair, flags, vert_scene);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_dcd_vf(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x,
                          const uint32_t* faces, const uint32_t* body, const float* vert_area, const float* face_area,
                          const float* d_hat, const float* offset, float kappa, lcs_pair* out, uint32_t out_capacity,
                          uint32_t* d_out_count, lcs_stream stream)
{
    if (!d_count || !x || !faces || !body || !vert_area || !face_area || !d_hat || !offset || !d_out_count ||
        (capacity && !pairs) || (out_capacity && !out))
        return lcs_fail(LCS_ERR_INVALID, "lcs_dcd_vf: bad argument");
    if (capacity == 0) return LCS_OK;
    k_dcd_vf<false><<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(pairs), d_count, capacity, reinterpret_cast<const float4*>(x),
        reinterpret_cast<const uint4*>(faces), body, vert_area, face_area, d_hat, offset, kappa, out, out_capacity,
        d_out_count, nullptr);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_dcd_ee(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x,
                          const uint32_t* edges, const uint32_t* body, const float* edge_area, const float* d_hat,
                          const float* offset, float kappa, lcs_pair* out, uint32_t out_capacity,
                          uint32_t* d_out_count, lcs_stream stream)
{
    if (!d_count || !x || !edges || !body || !edge_area || !d_hat || !offset || !d_out_count ||
        (capacity && !pairs) || (out_capacity && !out))
        return lcs_fail(LCS_ERR_INVALID, "lcs_dcd_ee: bad argument");
    if (capacity == 0) return LCS_OK;
    k_dcd_ee<false><<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(pairs), d_count, capacity, reinterpret_cast<const float4*>(x),
        reinterpret_cast<const uint2*>(edges), body, edge_area, d_hat, offset, kappa, out, out_capacity, d_out_count,
        nullptr);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

int lcs_dcd_vf_filtered(const uint32_t* ccd_pairs, const uint32_t* d_ccd_count, uint32_t capacity, const float* x,
                        const uint32_t* faces, const uint32_t* body, const float* vert_area, const float* face_area,
                        const float* d_hat, const float* offset, float kappa, lcs_pair* out, uint32_t out_capacity,
                        uint32_t* d_out_count, uint32_t* d_cand_count, lcs_stream stream)
{
    if (capacity == 0) return LCS_OK;
    k_dcd_vf<true><<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(ccd_pairs), d_ccd_count, capacity, reinterpret_cast<const float4*>(x),
        reinterpret_cast<const uint4*>(faces), body, vert_area, face_area, d_hat, offset, kappa, out, out_capacity,
        d_out_count, d_cand_count);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

int lcs_dcd_ee_filtered(const uint32_t* ccd_pairs, const uint32_t* d_ccd_count, uint32_t capacity, const float* x,
                        const uint32_t* edges, const uint32_t* body, const float* edge_area, const float* d_hat,
                        const float* offset, float kappa, lcs_pair* out, uint32_t out_capacity, uint32_t* d_out_count,
                        uint32_t* d_cand_count, lcs_stream stream)
{
    if (capacity == 0) return LCS_OK;
    k_dcd_ee<true><<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(ccd_pairs), d_ccd_count, capacity, reinterpret_cast<const float4*>(x),
        reinterpret_cast<const uint2*>(edges), body, edge_area, d_hat, offset, kappa, out, out_capacity, d_out_count,
        d_cand_count);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_contact_grad_diag(const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity, float* b,
                                     float* diag, lcs_stream stream)
{
    return grad_diag(pairs, d_count, capacity, b, diag, nullptr, stream);
}

extern "C" int lcs_contact_grad_diag_abd(const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity, float* b,
                                         float* diag, const lcs_abd_view* abd, lcs_stream stream)
{
    if (!abd) return lcs_fail(LCS_ERR_INVALID, "lcs_contact_grad_diag_abd: null view");
    return grad_diag(pairs, d_count, capacity, b, diag, abd, stream);
}

extern "C" int lcs_contact_energy(const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity, const float* x,
                                  const float* d_hat, const float* offset, double* d_energy, lcs_stream stream)
{
    if (!d_count || !x || !d_hat || !offset || !d_energy || (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_contact_energy: bad argument");
    if (capacity == 0) return LCS_OK;
    k_energy<<<grid_for(capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        pairs, d_count, capacity, reinterpret_cast<const float4*>(x), d_hat, offset, d_energy);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}
