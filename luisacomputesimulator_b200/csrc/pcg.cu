// pcg.cu -- 3x3 block SpMV and block-Jacobi preconditioned CG.
//
// Reference: ConjugateGradientSolver (Solver/LinearSolver/precond_cg.cpp:33-331, 626-771) and
// the SpMV NewtonSolver hands it (newton_solver.cpp:259-270, 347-472, 3397-3427).
//
// Two executions of the same recurrences:
//  * plain  -- the reference's dispatch structure: one kernel per operation (apply
//              preconditioner, its second pass, update p, SpMV, p.q, its second pass, step)
//              and a host read-back of r.z every `check_every` iterations;
//  * fused  -- one persistent cooperative launch for the whole solve: rows are owned by
//              threads, the three grid-wide reductions per iteration go through bounded
//              software grid barriers, and every block reduces the per-block partials in the
//              same fixed order, so all blocks agree on alpha / beta / convergence.
// Reductions are FP32 (the reference) or FP64 (precision form, LCS_PCG_FP64_DOTS).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include <mutex>
#include <new>

#include "lcs_common.cuh"
#include "lcs_internal.h"

using namespace lcs;

namespace {

constexpr float kPcgEps = 1e-10f;  // pcg_epsilon, precond_cg.cpp:12
constexpr int kFusedThreads = 1024; // one block per SM: 148 barrier participants / partial sums

__device__ __forceinline__ float safe_div(float a, float b) { return b < kPcgEps ? 0.0f : a / b; }

struct Bsr {
    const uint32_t* rp;
    const uint32_t* col;
    const float* val;
};

__device__ __forceinline__ float3 mv9(const float* __restrict__ m, float4 x)
{
    float3 y;
    y.x = __fmaf_rn(m[6], x.z, __fmaf_rn(m[3], x.y, m[0] * x.x));
    y.y = __fmaf_rn(m[7], x.z, __fmaf_rn(m[4], x.y, m[1] * x.x));
    y.z = __fmaf_rn(m[8], x.z, __fmaf_rn(m[5], x.y, m[2] * x.x));
    return y;
}

__device__ __forceinline__ float3 mv12(const float4* __restrict__ m, float4 x)
{
    const float4 c0 = m[0], c1 = m[1], c2 = m[2];
    float3 y;
    y.x = __fmaf_rn(c2.x, x.z, __fmaf_rn(c1.x, x.y, c0.x * x.x));
    y.y = __fmaf_rn(c2.y, x.z, __fmaf_rn(c1.y, x.y, c0.y * x.x));
    y.z = __fmaf_rn(c2.z, x.z, __fmaf_rn(c1.z, x.y, c0.z * x.x));
    return y;
}

// G lanes per row; returns the full row product on every lane of the group
template <int G>
__device__ __forceinline__ float3 row_product(uint32_t row, uint32_t lig, const float4* __restrict__ diag,
                                              const Bsr A, const Bsr B, const float4* x)
{
    float3 acc = make_float3(0.f, 0.f, 0.f);
    if (A.rp) {
        const uint32_t e = __ldg(&A.rp[row + 1]);
        for (uint32_t k = __ldg(&A.rp[row]) + lig; k < e; k += G) {
            const float3 t = mv9(A.val + 9 * (size_t)k, __ldcg(&x[__ldg(&A.col[k])]));
            acc.x += t.x; acc.y += t.y; acc.z += t.z;
        }
    }
    if (B.rp) {
        const uint32_t e = __ldcg(&B.rp[row + 1]);
        for (uint32_t k = __ldcg(&B.rp[row]) + lig; k < e; k += G) {
            const float3 t = mv9(B.val + 9 * (size_t)k, __ldcg(&x[__ldcg(&B.col[k])]));
            acc.x += t.x; acc.y += t.y; acc.z += t.z;
        }
    }
#pragma unroll
    for (int o = G >> 1; o > 0; o >>= 1) {
        acc.x += __shfl_xor_sync(0xFFFFFFFFu, acc.x, o);
        acc.y += __shfl_xor_sync(0xFFFFFFFFu, acc.y, o);
        acc.z += __shfl_xor_sync(0xFFFFFFFFu, acc.z, o);
    }
    const float3 d = mv12(diag + 3 * (size_t)row, __ldcg(&x[row]));
    return make_float3(d.x + acc.x, d.y + acc.y, d.z + acc.z);
}

template <int G>
__global__ void __launch_bounds__(256) k_spmv(uint32_t n, const float4* __restrict__ diag, Bsr A, Bsr B,
                                              const float4* x, float4* y)
{
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lig = gtid % G;
    const uint32_t ngroups = gridDim.x * blockDim.x / G;
    const uint32_t rows_round = (n + ngroups - 1) / ngroups * ngroups;
    for (uint32_t row = gtid / G; row < rows_round; row += ngroups) {
        const uint32_t r = row < n ? row : n - 1;  // whole groups stay converged for the shuffles
        const float3 v = row_product<G>(r, lig, diag, A, B, x);
        if (row < n && lig == 0) y[row] = make_float4(v.x, v.y, v.z, 0.0f);
    }
}

// ------------------------------------------------------------------------------------ plain
template <typename T>
__device__ __forceinline__ T block_sum(T v)
{
    __shared__ T red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane_id() == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    T s = 0;
    if (threadIdx.x == 0)
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) s += red[w];
    __syncthreads();
    return s;
}

// fn_pcg_init + fn_pcg_make_preconditioner (precond_cg.cpp:118-177, 256-267), x0 = 0
__global__ void k_plain_init(uint32_t n, const float4* __restrict__ b, const float4* __restrict__ diag, float4* x,
                             float4* r, float4* p, float4* minv, float* scal)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        r[i] = b[i];
        p[i] = make_float4(0, 0, 0, 0);
        x[i] = make_float4(0, 0, 0, 0);
        const float4 c0 = diag[3 * i], c1 = diag[3 * i + 1], c2 = diag[3 * i + 2];
        const float a = c0.x, bb = c1.x, c = c2.x, d = c0.y, e = c1.y, f = c2.y, g = c0.z, h = c1.z, k = c2.z;
        const float A = e * k - f * h, B = f * g - d * k, C = d * h - e * g;
        const float det = a * A + bb * B + c * C;
        const float id = 1.0f / det;
        minv[3 * i + 0] = make_float4(A * id, B * id, C * id, 0.0f);
        minv[3 * i + 1] = make_float4((c * h - bb * k) * id, (a * k - c * g) * id, (bb * g - a * h) * id, 0.0f);
        minv[3 * i + 2] = make_float4((bb * f - c * e) * id, (c * d - a * f) * id, (a * e - bb * d) * id, 0.0f);
    }
    if (blockIdx.x == 0 && threadIdx.x < 8) scal[threadIdx.x] = 0.0f;
}

// fn_pcg_apply_preconditioner (precond_cg.cpp:269-294): z = Minv r, partials of r.r and r.z
template <typename T>
__global__ void __launch_bounds__(256) k_plain_precond(uint32_t n, const float4* __restrict__ minv, const float4* r,
                                                       float4* z, T* part)
{
    T rr = 0, rz = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 rv = r[i];
        const float3 zv = mv12(minv + 3 * (size_t)i, rv);
        z[i] = make_float4(zv.x, zv.y, zv.z, 0.0f);
        rr += (T)__fmaf_rn(rv.z, rv.z, __fmaf_rn(rv.y, rv.y, rv.x * rv.x));
        rz += (T)__fmaf_rn(rv.z, zv.z, __fmaf_rn(rv.y, zv.y, rv.x * zv.x));
    }
    rr = block_sum(rr);
    rz = block_sum(rz);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rr;
        part[2 * blockIdx.x + 1] = rz;
    }
}

// fn_pcg_apply_preconditioner_second_pass (precond_cg.cpp:296-330): beta, r.z, |r| history.
// scal: 0 rr0, 1 rz, 2 alpha, 3 beta, 4 |r|, 5 |r0|, 6 nan flag
template <typename T>
__global__ void k_plain_precond2(const T* part, uint32_t nblocks, float* scal, int first)
{
    T rr = 0, rz = 0;
    for (uint32_t k = threadIdx.x; k < nblocks; k += blockDim.x) {
        rr += part[2 * k];
        rz += part[2 * k + 1];
    }
    rr = block_sum(rr);
    rz = block_sum(rz);
    if (threadIdx.x == 0) {
        const float frr = (float)rr, frz = (float)rz;
        scal[3] = safe_div(frz, scal[1]);
        scal[1] = frz;
        scal[4] = sqrtf(frr);
        if (first) scal[5] = sqrtf(frr);
    }
}

__global__ void k_plain_update_p(uint32_t n, const float4* z, float4* p, const float* scal)
{
    const float beta = scal[3];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 zv = z[i], pv = p[i];
        p[i] = make_float4(zv.x + beta * pv.x, zv.y + beta * pv.y, zv.z + beta * pv.z, 0.0f);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_plain_dot(uint32_t n, const float4* a, const float4* b, T* part)
{
    T s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 u = a[i], v = b[i];
        s += (T)__fmaf_rn(u.z, v.z, __fmaf_rn(u.y, v.y, u.x * v.x));
    }
    s = block_sum(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

template <typename T>
__global__ void k_plain_alpha(const T* part, uint32_t nblocks, float* scal)
{
    T s = 0;
    for (uint32_t k = threadIdx.x; k < nblocks; k += blockDim.x) s += part[k];
    s = block_sum(s);
    if (threadIdx.x == 0) scal[2] = safe_div(scal[1], (float)s);
}

// fn_pcg_step (precond_cg.cpp:240-253)
__global__ void k_plain_step(uint32_t n, float4* x, float4* r, const float4* p, const float4* q, const float* scal)
{
    const float alpha = scal[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 pv = p[i], qv = q[i], xv = x[i], rv = r[i];
        x[i] = make_float4(xv.x + alpha * pv.x, xv.y + alpha * pv.y, xv.z + alpha * pv.z, 0.0f);
        r[i] = make_float4(rv.x - alpha * qv.x, rv.y - alpha * qv.y, rv.z - alpha * qv.z, 0.0f);
    }
}

// -------------------------------------------------------------------------------- fused
struct FusedArgs {
    uint32_t n;
    const float4* diag;
    Bsr A, B;
    const float4* b;
    float4* x;
    float4 *r, *z, *p, *q, *minv;
    double* part;        // 3 * gridDim
    unsigned* bar_count;
    unsigned* bar_gen;
    int max_iter;
    float rel_tol, abs_rz_tol;
    int check_every;
    int fp64;
    lcs_pcg_stats* stats;
};

constexpr unsigned kBarrierSpinLimit = 1u << 24;

// software grid barrier for a cooperative launch; gives up (status LCS_ERR_TIMEOUT) after a
// bounded number of polls so that a stuck block can never hang the GPU
__device__ __forceinline__ bool grid_barrier(const FusedArgs& a, volatile int* s_fail)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = a.bar_gen;
        const unsigned g = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(a.bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            *a.bar_count = 0u;
            __threadfence();
            atomicAdd(a.bar_gen, 1u);
        } else {
            unsigned it = 0;
            while (*gen == g) {
                if (++it > kBarrierSpinLimit) {
                    *s_fail = 1;
                    a.stats->status = LCS_ERR_TIMEOUT;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *s_fail == 0;
}

// every block sums the per-block partials in the same order -> identical scalars everywhere
__device__ __forceinline__ void reduce_partials(const FusedArgs& a, int k, int count, double* out)
{
    __shared__ double s_out[3];
    if (threadIdx.x < 32) {
        double v[3] = {0.0, 0.0, 0.0};
        for (uint32_t b = threadIdx.x; b < gridDim.x; b += 32)
            for (int c = 0; c < count; ++c) v[c] += __ldcg(&a.part[3 * b + k + c]);
        for (int c = 0; c < count; ++c) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xFFFFFFFFu, v[c], o);
        }
        if (threadIdx.x == 0)
            for (int c = 0; c < count; ++c) s_out[c] = v[c];
    }
    __syncthreads();
    for (int c = 0; c < count; ++c) out[c] = s_out[c];
    __syncthreads();
}

template <int G>
__global__ void __launch_bounds__(kFusedThreads, 1) k_pcg_fused(FusedArgs a)
{
    __shared__ int s_fail;
    __shared__ double s_red[kFusedThreads / 32][3];
    if (threadIdx.x == 0) s_fail = 0;
    const uint32_t n = a.n;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;

    // x = 0, r = b, p = 0, Minv = inverse(D)
    for (uint32_t i = tid; i < n; i += nthreads) {
        a.r[i] = a.b[i];
        a.p[i] = make_float4(0, 0, 0, 0);
        a.x[i] = make_float4(0, 0, 0, 0);
        const float4 c0 = a.diag[3 * i], c1 = a.diag[3 * i + 1], c2 = a.diag[3 * i + 2];
        const float aa = c0.x, bb = c1.x, c = c2.x, d = c0.y, e = c1.y, f = c2.y, g = c0.z, h = c1.z, k = c2.z;
        const float A = e * k - f * h, B = f * g - d * k, C = d * h - e * g;
        const float id = 1.0f / (aa * A + bb * B + c * C);
        a.minv[3 * i + 0] = make_float4(A * id, B * id, C * id, 0.0f);
        a.minv[3 * i + 1] = make_float4((c * h - bb * k) * id, (aa * k - c * g) * id, (bb * g - aa * h) * id, 0.0f);
        a.minv[3 * i + 2] = make_float4((bb * f - c * e) * id, (c * d - aa * f) * id, (aa * e - bb * d) * id, 0.0f);
    }

    float rz_old = 0.0f, norm_r0 = 0.0f, norm_r = 0.0f, rz = 0.0f;
    int iter = 0, status = 0;
    for (iter = 0; iter < a.max_iter; ++iter) {
        // z = Minv r ; r.r ; r.z
        double rr_d = 0.0, rz_d = 0.0;
        float rr_f = 0.0f, rz_f = 0.0f;
        for (uint32_t i = tid; i < n; i += nthreads) {
            const float4 rv = a.r[i];
            const float3 zv = mv12(a.minv + 3 * (size_t)i, rv);
            a.z[i] = make_float4(zv.x, zv.y, zv.z, 0.0f);
            const float drr = __fmaf_rn(rv.z, rv.z, __fmaf_rn(rv.y, rv.y, rv.x * rv.x));
            const float drz = __fmaf_rn(rv.z, zv.z, __fmaf_rn(rv.y, zv.y, rv.x * zv.x));
            rr_d += drr; rz_d += drz; rr_f += drr; rz_f += drz;
        }
        {
            double v0 = a.fp64 ? rr_d : (double)rr_f, v1 = a.fp64 ? rz_d : (double)rz_f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                v0 += __shfl_xor_sync(0xFFFFFFFFu, v0, o);
                v1 += __shfl_xor_sync(0xFFFFFFFFu, v1, o);
            }
            if (lane_id() == 0) { s_red[threadIdx.x >> 5][0] = v0; s_red[threadIdx.x >> 5][1] = v1; }
            __syncthreads();
            if (threadIdx.x == 0) {
                double t0 = 0, t1 = 0;
                for (int w = 0; w < kFusedThreads / 32; ++w) { t0 += s_red[w][0]; t1 += s_red[w][1]; }
                a.part[3 * blockIdx.x + 0] = t0;
                a.part[3 * blockIdx.x + 1] = t1;
            }
        }
        if (!grid_barrier(a, &s_fail)) return;
        double red[2];
        reduce_partials(a, 0, 2, red);
        const float rr = (float)red[0];
        rz = (float)red[1];
        const float beta = safe_div(rz, rz_old);
        rz_old = rz;
        norm_r = sqrtf(rr);
        if (iter == 0) norm_r0 = norm_r;
        if (iter % a.check_every == 0) {
            if (isnan(rz) || isinf(rz)) { status = LCS_ERR_NAN; break; }
            if (rz < a.abs_rz_tol) break;
            if (a.rel_tol > 0.0f && norm_r <= a.rel_tol * norm_r0) break;
        }
        // p = z + beta p
        for (uint32_t i = tid; i < n; i += nthreads) {
            const float4 zv = a.z[i], pv = a.p[i];
            a.p[i] = make_float4(zv.x + beta * pv.x, zv.y + beta * pv.y, zv.z + beta * pv.z, 0.0f);
        }
        if (!grid_barrier(a, &s_fail)) return;
        // q = A p ; p.q
        double pq_d = 0.0;
        float pq_f = 0.0f;
        {
            const uint32_t lig = tid % G, ngroups = nthreads / G;
            const uint32_t rows_round = (n + ngroups - 1) / ngroups * ngroups;
            for (uint32_t row = tid / G; row < rows_round; row += ngroups) {
                const uint32_t rr_ = row < n ? row : n - 1;
                const float3 qv = row_product<G>(rr_, lig, a.diag, a.A, a.B, a.p);
                if (row < n && lig == 0) {
                    a.q[row] = make_float4(qv.x, qv.y, qv.z, 0.0f);
                    const float4 pv = __ldcg(&a.p[row]);
                    const float d = __fmaf_rn(pv.z, qv.z, __fmaf_rn(pv.y, qv.y, pv.x * qv.x));
                    pq_d += d;
                    pq_f += d;
                }
            }
            double v = a.fp64 ? pq_d : (double)pq_f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            if (lane_id() == 0) s_red[threadIdx.x >> 5][2] = v;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0;
                for (int w = 0; w < kFusedThreads / 32; ++w) t += s_red[w][2];
                a.part[3 * blockIdx.x + 2] = t;
            }
        }
        if (!grid_barrier(a, &s_fail)) return;
        double pq;
        reduce_partials(a, 2, 1, &pq);
        const float alpha = safe_div(rz, (float)pq);
        // x += alpha p ; r -= alpha q
        for (uint32_t i = tid; i < n; i += nthreads) {
            const float4 pv = a.p[i], qv = __ldcg(&a.q[i]), xv = a.x[i], rv = a.r[i];
            a.x[i] = make_float4(xv.x + alpha * pv.x, xv.y + alpha * pv.y, xv.z + alpha * pv.z, 0.0f);
            a.r[i] = make_float4(rv.x - alpha * qv.x, rv.y - alpha * qv.y, rv.z - alpha * qv.z, 0.0f);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.stats->iterations = iter;
        a.stats->rel_residual = norm_r0 > 0.0f ? norm_r / norm_r0 : 0.0f;
        a.stats->dot_rz = rz_old;
        if (a.stats->status == LCS_OK) a.stats->status = status;
    }
}

// ----------------------------------------------------------------------- row-resident solve
// One thread owns one block row for the whole solve: x, r, p and the inverted diagonal block
// live in registers, and only p crosses the grid (written once per iteration, gathered by
// the rows that reference it).  The material matrix is CSR or sliced ELL with 32-row slices
// (slot k of the 32 rows of a slice contiguous), which makes the thread-per-row loads of a
// warp coalesced.  Same recurrences, same stop rules and the same three grid-wide
// synchronisation points per iteration as k_pcg_fused.
struct RowArgs {
    uint32_t n;
    const float4* diag;
    int sell;              // material format: 0 CSR, 1 SELL-32
    const uint32_t* m_ptr; // CSR row_ptr (n + 1) | SELL slot offset of each slice (n_slices + 1, multiples of 4)
    const uint32_t* m_col; // CSR col | SELL col[(g * 32 + lane) * 4 + j], slot 4g + j (see row_matvec)
    const float* m_val;    // CSR 9 floats per block | SELL val[((g * 9 + c) * 32 + lane) * 4 + j]
    Bsr B;                 // contact blocks (CSR)
    int b_vec;             // B.val is 16-B aligned: contact values by 16-B loads
    const uint32_t* c_ptr; // the contact blocks again in SELL-32 (layout of m_*), or null
    const uint32_t* c_col;
    const float* c_val;
    const int* c_ok;       // device flag: the SELL copy is complete (else the CSR form is used)
    const float4* b;
    float4* x;
    float4* pg;            // p of every row, exchanged through L2
    double* part;          // 4 doubles per block
    unsigned* bar_count;
    unsigned* bar_gen;
    int max_iter;
    float rel_tol, abs_rz_tol;
    int check_every;
    int fp64;
    lcs_pcg_stats* stats;
};

__device__ __forceinline__ bool row_barrier(const RowArgs& a, volatile int* s_fail)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = a.bar_gen;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(a.bar_count, 1u) == gridDim.x - 1) {
            *a.bar_count = 0u;
            __threadfence();
            atomicAdd(a.bar_gen, 1u);
        } else {
            unsigned it = 0;
            while (*gen == g) {
                if (++it > kBarrierSpinLimit) {
                    *s_fail = 1;
                    a.stats->status = LCS_ERR_TIMEOUT;
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *s_fail == 0;
}

template <int BS>
__device__ __forceinline__ void block_partial(double v0, double v1, double* dst)
{
    __shared__ double s[BS / 32][2];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xFFFFFFFFu, v0, o);
        v1 += __shfl_xor_sync(0xFFFFFFFFu, v1, o);
    }
    if (lane_id() == 0) {
        s[threadIdx.x >> 5][0] = v0;
        s[threadIdx.x >> 5][1] = v1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
#pragma unroll
        for (int w = 0; w < BS / 32; ++w) {
            t0 += s[w][0];
            t1 += s[w][1];
        }
        dst[0] = t0;
        dst[1] = t1;
    }
}

// the same fixed-order sum of the per-block partials in every block
__device__ __forceinline__ void grid_sum(const double* part, int k, double& o0, double& o1)
{
    __shared__ double so[2];
    if (threadIdx.x < 32) {
        double v0 = 0.0, v1 = 0.0;
        for (uint32_t b = threadIdx.x; b < gridDim.x; b += 32) {
            v0 += __ldcg(&part[4 * b + k]);
            v1 += __ldcg(&part[4 * b + k + 1]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0 += __shfl_xor_sync(0xFFFFFFFFu, v0, o);
            v1 += __shfl_xor_sync(0xFFFFFFFFu, v1, o);
        }
        if (threadIdx.x == 0) {
            so[0] = v0;
            so[1] = v1;
        }
    }
    __syncthreads();
    o0 = so[0];
    o1 = so[1];
    __syncthreads();
}

__device__ __forceinline__ void acc_block(const float* m, int stride, float4 v, float& q0, float& q1, float& q2)
{
    q0 += __fmaf_rn(m[6 * stride], v.z, __fmaf_rn(m[3 * stride], v.y, m[0] * v.x));
    q1 += __fmaf_rn(m[7 * stride], v.z, __fmaf_rn(m[4 * stride], v.y, m[1 * stride] * v.x));
    q2 += __fmaf_rn(m[8 * stride], v.z, __fmaf_rn(m[5 * stride], v.y, m[2 * stride] * v.x));
}

// The 9 floats of contact block k in two steps, so that the loads of the next chunk can be issued
// before the current one is used: fetch_block9 issues three aligned 16-B loads covering the block
// (block k starts (k mod 4) floats into the 16-B word at 9k / 4) when the value array is 16-B aligned,
// else nine scalar loads (also for the array's last block, whose covering words may run past its end);
// block9 picks the 9 floats out.
struct Raw9 {
    float4 a, b, c;
    uint32_t sh;
};

__device__ __forceinline__ Raw9 fetch_block9(const float* val, uint32_t k, bool scalar)
{
    Raw9 r;
    if (scalar) {
        const float* m = val + 9 * (size_t)k;
        r.a = make_float4(__ldcg(m), __ldcg(m + 1), __ldcg(m + 2), __ldcg(m + 3));
        r.b = make_float4(__ldcg(m + 4), __ldcg(m + 5), __ldcg(m + 6), __ldcg(m + 7));
        r.c = make_float4(__ldcg(m + 8), 0.f, 0.f, 0.f);
        r.sh = 0;
    } else {
        const float4* v4 = reinterpret_cast<const float4*>(val) + ((9 * (size_t)k) >> 2);
        r.a = __ldcg(v4);
        r.b = __ldcg(v4 + 1);
        r.c = __ldcg(v4 + 2);
        r.sh = k & 3u;
    }
    return r;
}

__device__ __forceinline__ void block9(const Raw9& r, float m[9])
{
    const float w[12] = {r.a.x, r.a.y, r.a.z, r.a.w, r.b.x, r.b.y, r.b.z, r.b.w, r.c.x, r.c.y, r.c.z, r.c.w};
#pragma unroll
    for (int j = 0; j < 9; ++j) m[j] = r.sh == 0 ? w[j] : r.sh == 1 ? w[j + 1] : r.sh == 2 ? w[j + 2] : w[j + 3];
}

// Contact blocks of a warp's 32 consecutive rows r0 .. r0 + 31 (rows >= n have none), added to the
// calling lane's row accumulators (o0, o1, o2).  The rows' blocks form one CSR range, taken 32 blocks at
// a time with one block per lane (column, gather, values: neighbouring lanes read neighbouring blocks),
// summed per row by a segmented scan over the lanes and handed to the lane owning the row.  Columns are
// loaded two chunks ahead, gathers and values one chunk ahead of the chunk being summed.  Rows next to a prescribed
// boundary or inside a fold carry dozens of contact blocks; walking them one row per lane made every
// load of the warp touch 32 different lines.  Every lane of the warp must call this.
// Summation order: per chunk of 32 blocks a fixed tree, chunks in CSR order.
template <class LdU>
__device__ __forceinline__ void contact_warp(const Bsr& B, uint32_t r0, uint32_t n, bool vec, LdU ld_u, float& o0,
                                             float& o1, float& o2)
{
    const uint32_t lane = lane_id();
    const uint32_t total = __ldcg(&B.rp[n]);
    const uint32_t rp_l = __ldcg(&B.rp[min(r0 + lane, n)]);
    const uint32_t rend = __ldcg(&B.rp[min(r0 + 32u, n)]);
    const uint32_t rp_down = __shfl_down_sync(0xFFFFFFFFu, rp_l, 1);  // every lane takes part in each shuffle
    const uint32_t rp_next = lane < 31u ? rp_down : rend;
    const uint32_t kbeg = __shfl_sync(0xFFFFFFFFu, rp_l, 0);
    // software pipeline over the chunks: columns two chunks ahead, gathers and values one chunk ahead
    const uint32_t k0 = kbeg + lane;
    uint32_t col_a = k0 + 32u < rend ? __ldcg(&B.col[k0 + 32u]) : 0u;
    float4 u_cur = make_float4(0.f, 0.f, 0.f, 0.f);
    Raw9 raw{};
    if (k0 < rend) {
        u_cur = ld_u(__ldcg(&B.col[k0]));
        raw = fetch_block9(B.val, k0, !vec || k0 + 1u >= total);
    }
    for (uint32_t kc = kbeg; kc < rend; kc += 32u) {
        const uint32_t k = kc + lane;
        const bool act = k < rend;
        const uint32_t col_b = k + 64u < rend ? __ldcg(&B.col[k + 64u]) : 0u;
        float4 u_next = make_float4(0.f, 0.f, 0.f, 0.f);
        Raw9 raw_n{};
        if (k + 32u < rend) {
            u_next = ld_u(col_a);
            raw_n = fetch_block9(B.val, k + 32u, !vec || k + 33u >= total);
        }
        float y0 = 0.f, y1 = 0.f, y2 = 0.f;
        if (act) {
            const float4 v = u_cur;
            float m[9];
            block9(raw, m);
            y0 = __fmaf_rn(m[6], v.z, __fmaf_rn(m[3], v.y, m[0] * v.x));
            y1 = __fmaf_rn(m[7], v.z, __fmaf_rn(m[4], v.y, m[1] * v.x));
            y2 = __fmaf_rn(m[8], v.z, __fmaf_rn(m[5], v.y, m[2] * v.x));
        }
        // row (lane index) of block k: the last lane whose row starts at or before k
        uint32_t seg = 0;
#pragma unroll
        for (uint32_t st = 16; st > 0; st >>= 1) {
            const uint32_t cand = seg + st;
            const uint32_t v = __shfl_sync(0xFFFFFFFFu, rp_l, cand < 32u ? cand : 31u);
            if (cand < 32u && v <= k) seg = cand;
        }
        if (!act) seg = 32u + lane;  // past the range: a segment of its own
        // inclusive segmented scan: the last lane of each row's run holds the run's sum
#pragma unroll
        for (uint32_t d = 1; d < 32u; d <<= 1) {
            const float a0 = __shfl_up_sync(0xFFFFFFFFu, y0, d), a1 = __shfl_up_sync(0xFFFFFFFFu, y1, d),
                        a2 = __shfl_up_sync(0xFFFFFFFFu, y2, d);
            const uint32_t sg = __shfl_up_sync(0xFFFFFFFFu, seg, d);
            if (lane >= d && sg == seg) {
                y0 += a0;
                y1 += a1;
                y2 += a2;
            }
        }
        // this lane's row: its blocks in the chunk end at hi - 1
        const uint32_t lo = max(rp_l, kc), hi = min(min(rp_next, kc + 32u), rend);
        const bool mine = hi > lo;
        const uint32_t src = mine ? hi - 1u - kc : lane;
        const float s0 = __shfl_sync(0xFFFFFFFFu, y0, src), s1 = __shfl_sync(0xFFFFFFFFu, y1, src),
                    s2 = __shfl_sync(0xFFFFFFFFu, y2, src);
        if (mine) {
            o0 += s0;
            o1 += s1;
            o2 += s2;
        }
        col_a = col_b;
        u_cur = u_next;
        raw = raw_n;
    }
}

// streamed read-only 16-B load that does not displace L1 lines (matrix values: read once per iteration)
__device__ __forceinline__ float4 ld_stream4(const float4* p)
{
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
}

__device__ __forceinline__ float comp(const float4& v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }

// A v for the owned row: diagonal block + material (CSR or SELL) + contact (CSR).
//
// SELL material layout ("SELL-32, 4-slot groups"): a slice is 32 consecutive rows, its width (slots)
// padded to a multiple of 4; group g holds slots 4g..4g+3 of the 32 rows.  Column j of lane l is
// col[(g * 32 + l) * 4 + j] (one uint4 per lane), component c of slot j is
// val[((g * 9 + c) * 32 + l) * 4 + j] (one float4 per lane and component).  A warp therefore reads
// each group with one 512-B coalesced uint4 load and nine 512-B float4 loads, 2.5 load instructions per
// block instead of 10.  Padding slots hold zero blocks against the row itself.  The blocks are summed in
// slot order, the order of the CSR row.
// Groups [g0, g1) of a SELL-32 matrix (4-slot groups: columns col[(g * 32 + lane) * 4 + j], value
// component c at val[((g * 9 + c) * 32 + lane) * 4 + j]) against u, added to the lane's row sums in slot
// order.  Values are streamed past L1.
template <class LdU>
__device__ __forceinline__ void sell_range(const uint32_t* col, const float* val, uint32_t g0, uint32_t g1,
                                           uint32_t lane, LdU ld_u, float& o0, float& o1, float& o2)
{
    const uint4* C4 = reinterpret_cast<const uint4*>(col);
    const float4* V4 = reinterpret_cast<const float4*>(val);
    for (uint32_t g = g0; g < g1; ++g) {
        const uint4 jc = __ldg(&C4[(size_t)g * 32 + lane]);
        const float4 pv[4] = {ld_u(jc.x), ld_u(jc.y), ld_u(jc.z), ld_u(jc.w)};
        const float4* vg = V4 + (size_t)g * 9 * 32 + lane;
        // one output component at a time (block row r uses components r, r + 3, r + 6): three value
        // vectors live at once instead of nine
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const float4 ma = ld_stream4(vg + 32 * r), mb = ld_stream4(vg + 32 * (r + 3)), mc = ld_stream4(vg + 32 * (r + 6));
            float o = r == 0 ? o0 : r == 1 ? o1 : o2;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                o += __fmaf_rn(comp(mc, j), pv[j].z, __fmaf_rn(comp(mb, j), pv[j].y, comp(ma, j) * pv[j].x));
            if (r == 0) o0 = o;
            else if (r == 1) o1 = o;
            else o2 = o;
        }
    }
}

__device__ __forceinline__ void row_matvec(const RowArgs& a, uint32_t i, uint32_t row, bool own, uint32_t slice,
                                          uint32_t lane, const float4* src, float v0, float v1, float v2, float& q0,
                                          float& q1, float& q2)
{
    const float4 c0 = __ldg(&a.diag[3 * row]), c1 = __ldg(&a.diag[3 * row + 1]), c2 = __ldg(&a.diag[3 * row + 2]);
    q0 = __fmaf_rn(c2.x, v2, __fmaf_rn(c1.x, v1, c0.x * v0));
    q1 = __fmaf_rn(c2.y, v2, __fmaf_rn(c1.y, v1, c0.y * v0));
    q2 = __fmaf_rn(c2.z, v2, __fmaf_rn(c1.z, v1, c0.z * v0));
    float o0 = 0.f, o1 = 0.f, o2 = 0.f;
    const auto ld_src = [&](uint32_t col) { return __ldcg(&src[col]); };
    if (a.sell && slice * 32 < a.n) {  // threads past the last slice have no slot range
        sell_range(a.m_col, a.m_val, __ldg(&a.m_ptr[slice]) >> 2, __ldg(&a.m_ptr[slice + 1]) >> 2, lane, ld_src, o0,
                   o1, o2);
    } else if (a.m_ptr && own) {
        const uint32_t end = __ldg(&a.m_ptr[i + 1]);
        for (uint32_t k = __ldg(&a.m_ptr[i]); k < end; ++k)
            acc_block(a.m_val + 9 * (size_t)k, 1, __ldcg(&src[__ldg(&a.m_col[k])]), o0, o1, o2);
    }
    if (a.c_ptr && *a.c_ok) {
        if (slice * 32 < a.n)
            sell_range(a.c_col, a.c_val, __ldcg(&a.c_ptr[slice]) >> 2, __ldcg(&a.c_ptr[slice + 1]) >> 2, lane, ld_src,
                       o0, o1, o2);
    } else if (a.B.rp) {
        contact_warp(a.B, i - lane, a.n, a.b_vec != 0, ld_src, o0, o1, o2);
    }
    q0 += o0;
    q1 += o1;
    q2 += o2;
}

template <int BS>
__global__ void __launch_bounds__(BS) k_pcg_rows(RowArgs a)
{
    __shared__ int s_fail;
    if (threadIdx.x == 0) s_fail = 0;
    const uint32_t i = blockIdx.x * BS + threadIdx.x;
    const bool own = i < a.n;
    const uint32_t row = own ? i : a.n - 1;
    float x0 = 0.f, x1 = 0.f, x2 = 0.f, r0 = 0.f, r1 = 0.f, r2 = 0.f, p0 = 0.f, p1 = 0.f, p2 = 0.f;
    float m0, m1, m2, m3, m4, m5, m6, m7, m8;  // inverse diagonal block, column-major
    {
        const float4 bv = a.b[row];
        if (own) { r0 = bv.x; r1 = bv.y; r2 = bv.z; }
        const float4 c0 = a.diag[3 * row], c1 = a.diag[3 * row + 1], c2 = a.diag[3 * row + 2];
        const float aa = c0.x, bb = c1.x, c = c2.x, d = c0.y, e = c1.y, f = c2.y, g = c0.z, h = c1.z, k = c2.z;
        const float A = e * k - f * h, B = f * g - d * k, C = d * h - e * g;
        const float id = 1.0f / (aa * A + bb * B + c * C);
        m0 = A * id; m1 = B * id; m2 = C * id;
        m3 = (c * h - bb * k) * id; m4 = (aa * k - c * g) * id; m5 = (bb * g - aa * h) * id;
        m6 = (bb * f - c * e) * id; m7 = (c * d - aa * f) * id; m8 = (aa * e - bb * d) * id;
    }
    const uint32_t lane = threadIdx.x & 31u, slice = i >> 5;
    float rz_old = 0.0f, norm_r0 = 0.0f, norm_r = 0.0f;
    int iter = 0, status = 0;
    for (iter = 0; iter < a.max_iter; ++iter) {
        // z = Minv r ; r.r ; r.z
        const float z0 = __fmaf_rn(m6, r2, __fmaf_rn(m3, r1, m0 * r0));
        const float z1 = __fmaf_rn(m7, r2, __fmaf_rn(m4, r1, m1 * r0));
        const float z2 = __fmaf_rn(m8, r2, __fmaf_rn(m5, r1, m2 * r0));
        double drr, drz;
        if (a.fp64) {
            drr = (double)r0 * r0 + (double)r1 * r1 + (double)r2 * r2;
            drz = (double)r0 * z0 + (double)r1 * z1 + (double)r2 * z2;
        } else {
            drr = __fmaf_rn(r2, r2, __fmaf_rn(r1, r1, r0 * r0));
            drz = __fmaf_rn(r2, z2, __fmaf_rn(r1, z1, r0 * z0));
        }
        block_partial<BS>(drr, drz, &a.part[4 * blockIdx.x]);
        if (!row_barrier(a, &s_fail)) return;
        double srr, srz;
        grid_sum(a.part, 0, srr, srz);
        const float rr = (float)srr, rz = (float)srz;
        const float beta = safe_div(rz, rz_old);
        rz_old = rz;
        norm_r = sqrtf(rr);
        if (iter == 0) norm_r0 = norm_r;
        if (iter % a.check_every == 0) {
            if (isnan(rz) || isinf(rz)) { status = LCS_ERR_NAN; break; }
            if (rz < a.abs_rz_tol) break;
            if (a.rel_tol > 0.0f && norm_r <= a.rel_tol * norm_r0) break;
        }
        // p = z + beta p, published for the rows that reference it
        p0 = z0 + beta * p0;
        p1 = z1 + beta * p1;
        p2 = z2 + beta * p2;
        if (own) __stcg(&a.pg[i], make_float4(p0, p1, p2, 0.0f));
        if (!row_barrier(a, &s_fail)) return;
        // q = A p
        float q0, q1, q2;
        row_matvec(a, i, row, own, slice, lane, a.pg, p0, p1, p2, q0, q1, q2);
        double dpq;
        if (!own) dpq = 0.0;
        else if (a.fp64) dpq = (double)p0 * q0 + (double)p1 * q1 + (double)p2 * q2;
        else dpq = __fmaf_rn(p2, q2, __fmaf_rn(p1, q1, p0 * q0));
        block_partial<BS>(dpq, 0.0, &a.part[4 * blockIdx.x + 2]);
        if (!row_barrier(a, &s_fail)) return;
        double spq, unused;
        grid_sum(a.part, 2, spq, unused);
        const float alpha = safe_div(rz, (float)spq);
        x0 += alpha * p0; x1 += alpha * p1; x2 += alpha * p2;
        r0 -= alpha * q0; r1 -= alpha * q1; r2 -= alpha * q2;
    }
    if (own) a.x[i] = make_float4(x0, x1, x2, 0.0f);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.stats->iterations = iter;
        a.stats->rel_residual = norm_r0 > 0.0f ? norm_r / norm_r0 : 0.0f;
        a.stats->dot_rz = rz_old;
        if (a.stats->status == LCS_OK) a.stats->status = status;
    }
}

constexpr int kRowThreads = 256;

// ---------------------------------------------------------------- single-reduction row-resident solve
// Grid barrier, partial sums and their prefetch for the row-resident kernels.  The single-reduction
// form (Chronopoulos & Gear, "s-step iterative methods for symmetric linear systems", J. Comput.
// Appl. Math. 25, 1989) computes the same Krylov iterates as CG in exact arithmetic with the dot
// products of an iteration (r.u, w.u, r.r) in one grid-wide reduction.  With the block-Jacobi
// preconditioner M is row-local, so every vector but u stays with the thread that owns the row.
// Stop rules as in device_solve: r.z (= r.u) and |r| checked before the update.

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void red_add_release(unsigned* p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// grid barrier with release/acquire ordering (the block's writes, ordered by __syncthreads, are
// released by thread 0's arrival).  Thread 0 of each block tracks the barrier generation in `gen_seen`
// (read once at kernel start: no block can pass the first barrier before every block has arrived, so
// all read the same value), which saves a round trip per barrier.  Bounded spin -> LCS_ERR_TIMEOUT.
__device__ __forceinline__ bool pipe_barrier(unsigned* count, unsigned* gen, unsigned& gen_seen, lcs_pcg_stats* stats,
                                             volatile int* s_fail, unsigned spin_limit = kBarrierSpinLimit)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        if (atom_add_acq_rel(count, 1u) == gridDim.x - 1) {
            *count = 0u;  // ordered before the release below; no block arrives again before it
            red_add_release(gen, 1u);
        } else {
            unsigned it = 0;
            while (ld_acquire(gen) == gen_seen) {
                if (++it > spin_limit) {
                    *s_fail = 1;
                    stats->status = LCS_ERR_TIMEOUT;
                    break;
                }
            }
        }
        ++gen_seen;
    }
    __syncthreads();
    return *s_fail == 0;
}

template <int BS>
__device__ __forceinline__ void block_partial3(double v0, double v1, double v2, double* dst)
{
    __shared__ double s[BS / 32][3];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xFFFFFFFFu, v0, o);
        v1 += __shfl_xor_sync(0xFFFFFFFFu, v1, o);
        v2 += __shfl_xor_sync(0xFFFFFFFFu, v2, o);
    }
    if (lane_id() == 0) {
        s[threadIdx.x >> 5][0] = v0;
        s[threadIdx.x >> 5][1] = v1;
        s[threadIdx.x >> 5][2] = v2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
        for (int w = 0; w < BS / 32; ++w) {
            t0 += s[w][0];
            t1 += s[w][1];
            t2 += s[w][2];
        }
        dst[0] = t0;
        dst[1] = t1;
        dst[2] = t2;
    }
}

// Partial sums copied to shared memory by cp.async (no registers held while the SpMV runs): block b's
// four doubles land in dst[b]; grid_collect3 waits for the copies and reduces them in a fixed order.
constexpr int kPipeMaxBlocks = 448;  // 3 blocks on each of 148 SMs, rounded up

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}

template <int BS>
__device__ __forceinline__ void grid_prefetch3(const double* part, double (*dst)[4])
{
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += BS) {
        cp_async16(&dst[b][0], part + 4 * b);
        cp_async16(&dst[b][2], part + 4 * b + 2);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Grid-wide sums of the per-block partials, split in two so that the loads overlap other work:
// grid_fetch3 issues this thread's share of the loads (blocks t, t + BS, ... in that order),
// grid_reduce3 combines them in a fixed order (warp shuffles, then warps in index order).  Every
// block performs the same operations on the same data, so all get bit-identical sums.
struct Fetch3 {
    double v0, v1, v2;
};

template <int BS>
__device__ __forceinline__ Fetch3 grid_fetch3(const double* part)
{
    Fetch3 f{0.0, 0.0, 0.0};
#pragma unroll 2
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += BS) {
        f.v0 += __ldcg(&part[4 * b + 0]);
        f.v1 += __ldcg(&part[4 * b + 1]);
        f.v2 += __ldcg(&part[4 * b + 2]);
    }
    return f;
}

template <int BS>
__device__ __forceinline__ void grid_reduce3(Fetch3 f, double& o0, double& o1, double& o2);

template <int BS>
__device__ __forceinline__ void grid_collect3(double (*src)[4], double& o0, double& o1, double& o2)
{
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    Fetch3 f{0.0, 0.0, 0.0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += BS) {
        f.v0 += src[b][0];
        f.v1 += src[b][1];
        f.v2 += src[b][2];
    }
    grid_reduce3<BS>(f, o0, o1, o2);
}

template <int BS>
__device__ __forceinline__ void grid_reduce3(Fetch3 f, double& o0, double& o1, double& o2)
{
    __shared__ double s[BS / 32][3];
    __shared__ double so[3];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        f.v0 += __shfl_xor_sync(0xFFFFFFFFu, f.v0, o);
        f.v1 += __shfl_xor_sync(0xFFFFFFFFu, f.v1, o);
        f.v2 += __shfl_xor_sync(0xFFFFFFFFu, f.v2, o);
    }
    if (lane_id() == 0) {
        s[threadIdx.x >> 5][0] = f.v0;
        s[threadIdx.x >> 5][1] = f.v1;
        s[threadIdx.x >> 5][2] = f.v2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < BS / 32; ++w) t += s[w][threadIdx.x];
        so[threadIdx.x] = t;
    }
    __syncthreads();
    o0 = so[0];
    o1 = so[1];
    o2 = so[2];
    __syncthreads();
}

// Single-reduction row-resident solve (the Chronopoulos-Gear form of the same preconditioned CG):
// with w = A u and u = M^-1 r kept per row, gamma = r.u and delta = w.u are summed in ONE grid
// reduction, alpha = gamma / (delta - beta gamma / alpha_old), and p, s = A p, x, r follow by
// recurrence.  Two grid synchronisations per iteration (the reduction, and the publication of u
// before w = A u) instead of the three of k_pcg_rows; the only extra recurrence (s) keeps the
// rounding behaviour of the classic method, unlike fully pipelined forms, whose extra recurrences
// (A M^-1 w ...) drift apart in FP32 on stiff systems.
template <int BS>
__global__ void __launch_bounds__(BS, 3) k_pcg_cg1(RowArgs a)
{
    __shared__ int s_fail;
    // x, p, s of this block's rows: each read and written once per iteration, so they live in shared
    // memory (private slot per thread, no synchronisation) and leave registers to the SpMV
    __shared__ float4 sv[3][BS];
    __shared__ float4 sminv[3][BS];  // inverse diagonal block, column-major
    __shared__ __align__(16) double spart[kPipeMaxBlocks][4];  // every block's partial sums
    if (threadIdx.x == 0) s_fail = 0;
    unsigned gen_seen = threadIdx.x == 0 ? ld_acquire(a.bar_gen) : 0u;
    const uint32_t t = threadIdx.x;
#pragma unroll
    for (int k = 0; k < 3; ++k) sv[k][t] = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t i = blockIdx.x * BS + t;
    const bool own = i < a.n;
    const uint32_t row = own ? i : a.n - 1;
    const uint32_t lane = t & 31u, slice = i >> 5;
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    {
        const float4 bv = a.b[row];
        if (own) { r0 = bv.x; r1 = bv.y; r2 = bv.z; }
        const float4 c0 = a.diag[3 * row], c1 = a.diag[3 * row + 1], c2 = a.diag[3 * row + 2];
        const float aa = c0.x, bb = c1.x, c = c2.x, d = c0.y, e = c1.y, f = c2.y, g = c0.z, h = c1.z, k = c2.z;
        const float A = e * k - f * h, B = f * g - d * k, C = d * h - e * g;
        const float id = 1.0f / (aa * A + bb * B + c * C);
        sminv[0][t] = make_float4(A * id, B * id, C * id, 0.f);
        sminv[1][t] = make_float4((c * h - bb * k) * id, (aa * k - c * g) * id, (bb * g - aa * h) * id, 0.f);
        sminv[2][t] = make_float4((bb * f - c * e) * id, (c * d - aa * f) * id, (aa * e - bb * d) * id, 0.f);
    }
#define LCS_MINV(v0, v1, v2, o0, o1, o2)                                                 \
    {                                                                                     \
        const float4 mc0 = sminv[0][t], mc1 = sminv[1][t], mc2 = sminv[2][t];             \
        o0 = __fmaf_rn(mc2.x, v2, __fmaf_rn(mc1.x, v1, mc0.x * v0));                      \
        o1 = __fmaf_rn(mc2.y, v2, __fmaf_rn(mc1.y, v1, mc0.y * v0));                      \
        o2 = __fmaf_rn(mc2.z, v2, __fmaf_rn(mc1.z, v1, mc0.z * v0));                      \
    }
    float u0, u1, u2, w0, w1, w2;
    LCS_MINV(r0, r1, r2, u0, u1, u2)
    // u is published before every w = A u; the reduction barrier between a SpMV and the next
    // publication guarantees every block has finished reading, so one buffer suffices
    if (own) __stcg(&a.pg[i], make_float4(u0, u1, u2, 0.0f));
    if (!pipe_barrier(a.bar_count, a.bar_gen, gen_seen, a.stats, &s_fail)) return;
    row_matvec(a, i, row, own, slice, lane, a.pg, u0, u1, u2, w0, w1, w2);
    float gamma_old = 0.0f, alpha_old = 0.0f, norm_r0 = 0.0f, norm_r = 0.0f, gamma = 0.0f;
    int iter = 0, status = 0;
    for (iter = 0; iter < a.max_iter; ++iter) {
        double dg, dd, dr;
        if (a.fp64) {
            dg = (double)r0 * u0 + (double)r1 * u1 + (double)r2 * u2;
            dd = (double)w0 * u0 + (double)w1 * u1 + (double)w2 * u2;
            dr = (double)r0 * r0 + (double)r1 * r1 + (double)r2 * r2;
        } else {
            dg = __fmaf_rn(r2, u2, __fmaf_rn(r1, u1, r0 * u0));
            dd = __fmaf_rn(w2, u2, __fmaf_rn(w1, u1, w0 * u0));
            dr = __fmaf_rn(r2, r2, __fmaf_rn(r1, r1, r0 * r0));
        }
        if (!own) dg = dd = dr = 0.0;
        double* part = a.part + 4 * (size_t)gridDim.x * (iter & 1);
        block_partial3<BS>(dg, dd, dr, &part[4 * blockIdx.x]);
        if (!pipe_barrier(a.bar_count, a.bar_gen, gen_seen, a.stats, &s_fail)) return;
        grid_prefetch3<BS>(part, spart);
        double sg, sd, sr;
        grid_collect3<BS>(spart, sg, sd, sr);
        gamma = (float)sg;
        const float delta = (float)sd;
        norm_r = sqrtf((float)sr);
        if (iter == 0) norm_r0 = norm_r;
        if (iter % a.check_every == 0) {
            if (isnan(gamma) || isinf(gamma)) { status = LCS_ERR_NAN; break; }
            if (gamma < a.abs_rz_tol) break;
            if (a.rel_tol > 0.0f && norm_r <= a.rel_tol * norm_r0) break;
        }
        // p.Ap = delta - beta gamma / alpha_old can cancel to below pcg_epsilon near convergence;
        // the iteration then restarts from the current residual (beta = 0, p = u), as on the first
        float beta = 0.0f, alpha = 0.0f;
        bool restart = iter == 0 || alpha_old == 0.0f;
        if (!restart) {
            beta = safe_div(gamma, gamma_old);
            const float den = delta - beta * gamma / alpha_old;
            restart = !(den >= kPcgEps);
            if (!restart) alpha = gamma / den;
        }
        if (restart) {
            beta = 0.0f;
            alpha = safe_div(gamma, delta);
        }
        float4 sd4 = sv[2][t], p = sv[1][t], x = sv[0][t];
        p = make_float4(u0 + beta * p.x, u1 + beta * p.y, u2 + beta * p.z, 0.f);
        sd4 = make_float4(w0 + beta * sd4.x, w1 + beta * sd4.y, w2 + beta * sd4.z, 0.f);
        x = make_float4(x.x + alpha * p.x, x.y + alpha * p.y, x.z + alpha * p.z, 0.f);
        sv[2][t] = sd4; sv[1][t] = p; sv[0][t] = x;
        r0 -= alpha * sd4.x; r1 -= alpha * sd4.y; r2 -= alpha * sd4.z;
        LCS_MINV(r0, r1, r2, u0, u1, u2)
        if (own) __stcg(&a.pg[i], make_float4(u0, u1, u2, 0.0f));
        if (!pipe_barrier(a.bar_count, a.bar_gen, gen_seen, a.stats, &s_fail)) return;
        row_matvec(a, i, row, own, slice, lane, a.pg, u0, u1, u2, w0, w1, w2);
        gamma_old = gamma;
        alpha_old = alpha;
    }
#undef LCS_MINV
    if (own) a.x[i] = sv[0][t];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.stats->iterations = iter;
        a.stats->rel_residual = norm_r0 > 0.0f ? norm_r / norm_r0 : 0.0f;
        a.stats->dot_rz = gamma;
        if (a.stats->status == LCS_OK) a.stats->status = status;
    }
}

// ------------------------------------------------------------ slice-resident single-reduction solve
// The same single-reduction PCG as k_pcg_cg1 for a SELL-32 material matrix, laid out for one block per
// SM: block c owns the contiguous slices [c S / P, (c + 1) S / P) (S slices, P blocks), so every SM
// holds the same number of rows (within one slice).  Per solve the block copies the first `gres` 4-slot
// groups of each of its slices (values and columns) into shared memory, where they stay for all
// iterations; the remaining groups, the diagonal and the contact blocks are read from L2 as before.
// u of the block's own rows is kept in shared memory too, so only columns owned by other blocks are
// gathered from L2.
//
// Synchronisation: the dot-product reduction is a grid barrier; the publication of u before w = A u
// is not -- each block waits only for the blocks whose rows its own rows reference (a bit mask built
// once per solve from the material and contact columns), through per-block flags holding the
// iteration each block last published.  A block overwrites u only after the next reduction barrier,
// which every reader of the previous u has passed, so one u buffer suffices (as in k_pcg_cg1).
// Summation orders are those of k_pcg_cg1: the diagonal, the material slots in slot order, the
// contact blocks in CSR order; the dot products in a fixed order over warps and blocks.
constexpr int kResThreads = 640;                           // at most 20 slices (640 rows) per block
constexpr int kResGroupBytes = 9 * 32 * 16 + 32 * 16;      // values + columns of one group of a slice
// contact blocks of a block's rows are multiplied by all its threads, kResContactChunk at a time, the products
// kept in shared memory (3 floats each) for the rows' owners
constexpr int kResContactChunk = 1536;
constexpr int kResMaxBlocks = 512;
constexpr int kResDepWords = kResMaxBlocks / 32;

struct ResArgs {
    RowArgs a;
    const uint32_t* part;   // P + 1: block c owns slices [part[c], part[c + 1])
    const uint32_t* owner;  // S: the block owning each slice
    unsigned* flags;     // per block: the last iteration tag whose u the block published
    uint32_t n_slices;
    uint32_t max_slices; // slices of the largest block (shared-memory stride)
    int gres;            // resident groups per slice
    int gtm;             // further groups per slice held in tensor memory (0: none)
};

// Tensor memory (TMEM, 256 KB per SM) as on-chip storage for the material groups beyond the shared-memory ones:
// warp w of the block reaches TMEM lanes 32 (w mod 4) .. 32 (w mod 4) + 31, one per thread, and keeps its slice's
// groups there, 40 columns each (the group's column word, then its nine value words), from column 80 (w / 4),
// and the lanes' diagonal blocks (three float4 columns, 12 words) from column 400 + 12 (w / 4).  With at most
// 20 warps that is columns 0..459 of the 512 the block allocates.
constexpr int kResTmemGroups = 2;
constexpr uint32_t kResTmemCols = 512;
__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, uint32_t ncols)
{
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint4 v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(v.x), "r"(v.y),
                 "r"(v.z), "r"(v.w)
                 : "memory");
}
__device__ __forceinline__ uint4 tmem_ld4(uint32_t taddr)
{
    uint4 v;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(taddr)
                 : "memory");
    return v;
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ float4 as_f4(uint4 v)
{
    return make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z), __uint_as_float(v.w));
}
__device__ __forceinline__ uint4 as_u4(float4 v)
{
    return make_uint4(__float_as_uint(v.x), __float_as_uint(v.y), __float_as_uint(v.z), __float_as_uint(v.w));
}

// Slices to blocks by cost, before each solve: a slice costs its material groups, its contact blocks (CSR)
// and kResSliceBase for the diagonal and the vectors; block c takes the slices whose cost prefix reaches
// c / P of the total, with at most `cap` slices per block and at least one, and every later block still
// able to take the rest.  One block of 1024 threads: the prefix by block scans, the ideal cuts by one
// binary search per block, the clamping in one thread.
// Cost weights of a slice's work (compile-time), fitted to per-block A u times measured on the 88,800-row
// tube system (about 0.02 us per slice, 0.04 per material group, 0.004 per contact block, whose gathers
// are scattered): material groups held in shared memory (the first `gres` of the slice), material groups
// read from L2, contact blocks (per 16), and the diagonal and vectors.
#ifndef LCS_RES_W_SMEM
#define LCS_RES_W_SMEM 4
#endif
#ifndef LCS_RES_W_L2
#define LCS_RES_W_L2 4
#endif
#ifndef LCS_RES_W_CONTACT
#define LCS_RES_W_CONTACT 4
#endif
#ifndef LCS_RES_SLICE_BASE
#define LCS_RES_SLICE_BASE 8
#endif
constexpr uint32_t kResSliceBase = LCS_RES_SLICE_BASE;
constexpr uint32_t kResMaxSlices = kResMaxBlocks * (kResThreads / 32);  // the partition's shared prefix

__global__ void __launch_bounds__(1024) k_res_partition(uint32_t S, uint32_t P, uint32_t cap, const uint32_t* __restrict__ m_ptr,
                                                        const uint32_t* __restrict__ c_rp, uint32_t n,
                                                        uint32_t* __restrict__ part, uint32_t* __restrict__ owner,
                                                        uint32_t gres)
{
    __shared__ uint32_t prefix[kResMaxSlices + 1];  // cost of slices [0, s)
    __shared__ uint32_t cut[kResMaxBlocks + 1];
    __shared__ uint32_t ws[32];
    __shared__ uint32_t carry;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    if (t == 0) carry = 0u;
    __syncthreads();
    for (uint32_t base = 0; base < S; base += 1024u) {
        const uint32_t sl = base + t;
        uint32_t v = 0u;
        if (sl < S) {
            const uint32_t mg = (m_ptr[sl + 1] - m_ptr[sl]) >> 2, ms = mg < gres ? mg : gres;
            v = LCS_RES_W_SMEM * ms + LCS_RES_W_L2 * (mg - ms) + kResSliceBase;
            if (c_rp) v += (LCS_RES_W_CONTACT * (c_rp[min(32u * sl + 32u, n)] - c_rp[32u * sl])) >> 4;
        }
        uint32_t incl = v;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += x;
        }
        if (lane == 31u) ws[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = ws[lane];
#pragma unroll
            for (uint32_t o = 1; o < 32u; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= o) w += x;
            }
            ws[lane] = w;
        }
        __syncthreads();
        if (sl < S) prefix[sl] = carry + (warp ? ws[warp - 1] : 0u) + incl - v;
        __syncthreads();
        if (t == 0) carry += ws[31];
        __syncthreads();
    }
    if (t == 0) prefix[S] = carry;
    __syncthreads();
    const uint64_t total = carry;
    // ideal cut of block c: the first slice whose prefix reaches c / P of the total
    for (uint32_t c = t; c <= P; c += 1024u) {
        const uint64_t target = total * c / P;
        uint32_t lo = 0, hi = S;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if ((uint64_t)prefix[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        cut[c] = lo;
    }
    __syncthreads();
    if (t == 0) {
        uint32_t prev = 0u;
        cut[0] = 0u;
        for (uint32_t c = 1; c < P; ++c) {
            const uint32_t lo = max(prev + 1u, S > cap * (P - c) ? S - cap * (P - c) : 0u);
            const uint32_t hi = min(prev + cap, S - (P - c));
            const uint32_t b = min(max(cut[c], lo), hi);
            cut[c] = b;
            prev = b;
        }
        cut[P] = S;
    }
    __syncthreads();
    for (uint32_t c = t; c <= P; c += 1024u) part[c] = cut[c];
    for (uint32_t c = warp; c < P; c += 32u)
        for (uint32_t sl = cut[c] + lane; sl < cut[c + 1]; sl += 32u) owner[sl] = c;
}

__device__ __forceinline__ void st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// publish this block's u (stores already issued by every thread), then wait for the blocks in `dep`:
// thread b waits for block b, so all waits run at once.  Flags are kResFlagStride words apart (one
// 32-B sector each), so the polls of different blocks do not share a sector.
constexpr int kResFlagStride = 8;

__device__ __forceinline__ bool res_publish_wait(unsigned* flags, unsigned tag, const unsigned* dep,
                                                 lcs_pcg_stats* stats, volatile int* s_fail,
                                                 unsigned spin_limit = kBarrierSpinLimit)
{
    __syncthreads();
    const uint32_t t = threadIdx.x;
    if (t == 0) st_release(flags + kResFlagStride * blockIdx.x, tag);  // releases the block's u, ordered by the barrier
    if (t < gridDim.x && ((dep[t >> 5] >> (t & 31u)) & 1u)) {
        const unsigned* f = flags + kResFlagStride * t;
        unsigned it = 0;
        while ((int)(ld_acquire(f) - tag) < 0) {
            if (++it > spin_limit) {
                *s_fail = 1;
                stats->status = LCS_ERR_TIMEOUT;
                break;
            }
        }
    }
    __syncthreads();
    return *s_fail == 0;
}

// Grid-wide sums of the blocks' three partials without a counter barrier: block c stores its partials
// tagged with the iteration (the low four mantissa bits of each double set to iter mod 15; 15 marks an
// empty slot, the host fills the buffers with it before a solve), every block polls the 3 P slots of the
// iteration's buffer until each carries the tag, clears the tag bits and sums the partials in block order
// (the same sums in every block).  Slots alternate between two buffers by iteration parity: a block can
// only rewrite a buffer after every block has read it, since its next partial needs the next iteration's
// sums, which need every block's next partial, which each block writes only after reading this one.
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
constexpr unsigned long long kTagMask = 0xFull;

template <int BT>
__device__ __forceinline__ bool res_allgather3(double v0, double v1, double v2, unsigned long long* part, unsigned tag,
                                               double (*spart)[4], lcs_pcg_stats* stats, volatile int* s_fail,
                                               double& o0, double& o1, double& o2,
                                               unsigned spin_limit = kBarrierSpinLimit)
{
    __shared__ double s[BT / 32][3];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xFFFFFFFFu, v0, o);
        v1 += __shfl_xor_sync(0xFFFFFFFFu, v1, o);
        v2 += __shfl_xor_sync(0xFFFFFFFFu, v2, o);
    }
    if (lane_id() == 0) {
        s[threadIdx.x >> 5][0] = v0;
        s[threadIdx.x >> 5][1] = v1;
        s[threadIdx.x >> 5][2] = v2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
        for (int w = 0; w < BT / 32; ++w) {
            t0 += s[w][0];
            t1 += s[w][1];
            t2 += s[w][2];
        }
        unsigned long long* dst = part + 4 * (size_t)blockIdx.x;
        st_relaxed_u64(dst + 0, ((unsigned long long)__double_as_longlong(t0) & ~kTagMask) | tag);
        st_relaxed_u64(dst + 1, ((unsigned long long)__double_as_longlong(t1) & ~kTagMask) | tag);
        st_relaxed_u64(dst + 2, ((unsigned long long)__double_as_longlong(t2) & ~kTagMask) | tag);
    }
    for (uint32_t k = threadIdx.x; k < 3 * gridDim.x; k += BT) {
        const unsigned long long* src = part + 4 * (size_t)(k / 3) + k % 3;
        unsigned long long bits;
        unsigned it = 0;
        while (((bits = ld_relaxed_u64(src)) & kTagMask) != tag) {
            if (++it > spin_limit) {
                *s_fail = 1;
                stats->status = LCS_ERR_TIMEOUT;
                break;
            }
        }
        spart[k / 3][k % 3] = __longlong_as_double((long long)(bits & ~kTagMask));
    }
    __syncthreads();
    if (*s_fail) return false;
    Fetch3 f{0.0, 0.0, 0.0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += BT) {
        f.v0 += spart[b][0];
        f.v1 += spart[b][1];
        f.v2 += spart[b][2];
    }
    grid_reduce3<BT>(f, o0, o1, o2);
    return true;
}

// The two bounded waits of the slice-resident solve (the tagged reduction and the neighbour-flag wait)
// with a wait that nothing satisfies: block `missing` neither arrives nor publishes, so every other block
// must give up after spin_limit polls and report LCS_ERR_TIMEOUT (missing < 0: every block takes part and
// the waits complete).  Each block waits for every other one.
__global__ void k_wait_probe(int which, int missing, unsigned spin_limit, unsigned long long* part,
                             unsigned* flags, lcs_pcg_stats* stats)
{
    __shared__ int s_fail;
    __shared__ unsigned s_dep[kResDepWords];
    __shared__ double spart[32][4];
    if (threadIdx.x == 0) s_fail = 0;
    for (uint32_t w = threadIdx.x; w < (uint32_t)kResDepWords; w += blockDim.x) {
        unsigned m = 0u;
        for (uint32_t b = 32 * w; b < 32 * w + 32 && b < gridDim.x; ++b)
            if (b != blockIdx.x) m |= 1u << (b & 31u);
        s_dep[w] = m;
    }
    __syncthreads();
    if ((int)blockIdx.x == missing) return;
    if (which == 0) {
        double o0, o1, o2;
        res_allgather3<128>(1.0, 2.0, 3.0, part, 0u, spart, stats, &s_fail, o0, o1, o2, spin_limit);
    } else {
        res_publish_wait(flags, 1u, s_dep, stats, &s_fail, spin_limit);
    }
}

template <int BT>
__global__ void __launch_bounds__(BT, 1) k_pcg_res(ResArgs ra)
{
    const RowArgs& a = ra.a;
    extern __shared__ __align__(16) unsigned char res_smem[];
    __shared__ int s_fail;
    __shared__ unsigned s_dep[kResDepWords];
    __shared__ uint32_t s_taddr;
    const uint32_t P = gridDim.x, c = blockIdx.x;
    const uint32_t s_lo = __ldcg(&ra.part[c]), s_hi = __ldcg(&ra.part[c + 1]);
    const uint32_t nsl = s_hi - s_lo, row0 = 32u * s_lo;
    const int G = ra.gres;
    const int GT = ra.gtm;
    float* cprod = reinterpret_cast<float*>(res_smem);                     // [3][kResContactChunk]
    double(*spart)[4] = reinterpret_cast<double(*)[4]>(cprod + 3 * kResContactChunk);  // P
    float4* sval = reinterpret_cast<float4*>(spart + P);                   // [max_slices * G][9][32]
    uint4* scol = reinterpret_cast<uint4*>(sval + (size_t)ra.max_slices * G * 9 * 32);  // [max_slices * G][32]
    const uint32_t t = threadIdx.x, ls = t >> 5, lane = t & 31u;
    const uint32_t i = row0 + t;
    const bool own = ls < nsl && i < a.n;
    const uint32_t row = own ? i : row0;
    const uint32_t slice = s_lo + ls;
    if (t == 0) s_fail = 0;
    for (int w = t; w < kResDepWords; w += BT) s_dep[w] = 0u;
    const uint4* C4 = reinterpret_cast<const uint4*>(a.m_col);
    const float4* V4 = reinterpret_cast<const float4*>(a.m_val);
    uint32_t g0 = 0, g1 = 0;
    if (ls < nsl) {
        g0 = __ldg(&a.m_ptr[slice]) >> 2;
        g1 = __ldg(&a.m_ptr[slice + 1]) >> 2;
        // this warp's slice: resident groups to shared memory
        const uint32_t nres = min((uint32_t)G, g1 - g0);
        for (uint32_t j = 0; j < nres; ++j) {
            const float4* src = V4 + (size_t)(g0 + j) * 9 * 32;
            float4* dst = sval + ((size_t)ls * G + j) * 9 * 32;
#pragma unroll
            for (int k = 0; k < 9; ++k) dst[32 * k + lane] = ld_stream4(src + 32 * k + lane);
            scol[((size_t)ls * G + j) * 32 + lane] = __ldg(&C4[(size_t)(g0 + j) * 32 + lane]);
        }
    }
    if (GT > 0) {
        if (ls == 0) tmem_alloc(&s_taddr, kResTmemCols);
        tmem_fence_before();
    }
    __syncthreads();  // s_dep cleared, tensor memory allocated
    // this warp's slice: the next GT groups to tensor memory (warp-uniform: every lane of the warp takes part)
    uint32_t tbase = 0;
    if (GT > 0) {
        tmem_fence_after();
        tbase = s_taddr + ((32u * (ls & 3u)) << 16) + 80u * (ls >> 2);
        if (ls < nsl && g1 - g0 > (uint32_t)G) {
            const uint32_t nt = min((uint32_t)GT, g1 - g0 - (uint32_t)G);
            for (uint32_t jt = 0; jt < nt; ++jt) {
                const uint32_t g = g0 + (uint32_t)G + jt;
                const uint32_t cb = tbase + 40u * jt;
                tmem_st4(cb, __ldg(&C4[(size_t)g * 32 + lane]));
#pragma unroll
                for (int k = 0; k < 9; ++k) tmem_st4(cb + 4u + 4u * k, as_u4(ld_stream4(V4 + ((size_t)g * 9 + k) * 32 + lane)));
            }
        }
        if (ls < nsl) {  // the diagonal blocks of the warp's rows
            const uint32_t db = s_taddr + ((32u * (ls & 3u)) << 16) + 400u + 12u * (ls >> 2);
#pragma unroll
            for (int k = 0; k < 3; ++k) tmem_st4(db + 4u * k, as_u4(__ldg(&a.diag[3 * row + k])));
        }
        tmem_wait_st();
    }
    // the blocks this block's rows read u from: a window of 32 blocks around c by warp vote, others
    // (distant contacts) one shared-memory OR each
    {
        unsigned near = 0u;
        auto note = [&](uint32_t col) {
            const uint32_t oc = __ldcg(&ra.owner[col >> 5]);
            if (oc == c) return;
            const int d = (int)oc - (int)c + 16;
            if (d >= 0 && d < 32) near |= 1u << d;
            else atomicOr(&s_dep[oc >> 5], 1u << (oc & 31u));
        };
        if (ls < nsl) {
            for (uint32_t g = g0; g < g1; ++g) {
                const uint4 jc = __ldg(&C4[(size_t)g * 32 + lane]);
                if (own) { note(jc.x); note(jc.y); note(jc.z); note(jc.w); }
            }
        }
        if (a.B.rp && own) {
            const uint32_t end = __ldcg(&a.B.rp[i + 1]);
            for (uint32_t k = __ldcg(&a.B.rp[i]); k < end; ++k) note(__ldcg(&a.B.col[k]));
        }
        near = __reduce_or_sync(0xFFFFFFFFu, near);
        if (lane == 0) {
            while (near) {
                const int d = __ffs(near) - 1;
                near &= near - 1u;
                const uint32_t oc = c + (uint32_t)d - 16u;
                atomicOr(&s_dep[oc >> 5], 1u << (oc & 31u));
            }
        }
    }
    // u = M^-1 b; the inverse diagonal block stays in registers
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    float m0, m1, m2, m3, m4, m5, m6, m7, m8;
    {
        const float4 bv = a.b[row];
        if (own) { r0 = bv.x; r1 = bv.y; r2 = bv.z; }
        const float4 c0 = a.diag[3 * row], c1 = a.diag[3 * row + 1], c2 = a.diag[3 * row + 2];
        const float aa = c0.x, bb = c1.x, cc = c2.x, d = c0.y, e = c1.y, f = c2.y, g = c0.z, h = c1.z, k = c2.z;
        const float A = e * k - f * h, B = f * g - d * k, C = d * h - e * g;
        const float id = 1.0f / (aa * A + bb * B + cc * C);
        m0 = A * id; m1 = B * id; m2 = C * id;
        m3 = (cc * h - bb * k) * id; m4 = (aa * k - cc * g) * id; m5 = (bb * g - aa * h) * id;
        m6 = (bb * f - cc * e) * id; m7 = (cc * d - aa * f) * id; m8 = (aa * e - bb * d) * id;
    }
    // the contact blocks of the block's rows, [ce0, ce1) of the CSR, and of the lane's row (fixed for the solve)
    const uint32_t row_end = min(32u * s_hi, a.n);
    const uint32_t ce0 = a.B.rp ? __ldcg(&a.B.rp[row0]) : 0u, ce1 = a.B.rp ? __ldcg(&a.B.rp[row_end]) : 0u;
    const uint32_t re0 = a.B.rp && own ? __ldcg(&a.B.rp[i]) : 0u, re1 = a.B.rp && own ? __ldcg(&a.B.rp[i + 1]) : 0u;
    const bool c_vec = a.b_vec != 0;
    const uint32_t c_total = a.B.rp ? __ldcg(&a.B.rp[a.n]) : 0u;
    auto ld_u = [&](uint32_t col) -> float4 { return __ldcg(&a.pg[col]); };
    // contact blocks [k0, k0 + cnt) times u, one block per thread, into shared memory
    // the column of the thread's first contact block, fixed for the solve, stays in a register
    const uint32_t c_col0 = t < ce1 - ce0 ? __ldcg(&a.B.col[ce0 + t]) : 0u;
    auto contact_chunk = [&](uint32_t k0, uint32_t cnt) {
        for (uint32_t k = t; k < cnt; k += BT) {
            const uint32_t e = k0 + k;
            const float4 v = ld_u(e == ce0 + t ? c_col0 : __ldcg(&a.B.col[e]));
            float m[9];
            block9(fetch_block9(a.B.val, e, !c_vec || e + 1u >= c_total), m);
            cprod[k] = __fmaf_rn(m[6], v.z, __fmaf_rn(m[3], v.y, m[0] * v.x));
            cprod[kResContactChunk + k] = __fmaf_rn(m[7], v.z, __fmaf_rn(m[4], v.y, m[1] * v.x));
            cprod[2 * kResContactChunk + k] = __fmaf_rn(m[8], v.z, __fmaf_rn(m[5], v.y, m[2] * v.x));
        }
    };
    // the products of chunk [k0, k0 + cnt) that belong to the lane's row, in CSR order
    auto contact_add = [&](uint32_t k0, uint32_t cnt, float& o0, float& o1, float& o2) {
        const uint32_t lo = max(re0, k0), hi = min(re1, k0 + cnt);
        for (uint32_t e = lo; e < hi; ++e) {
            o0 += cprod[e - k0];
            o1 += cprod[kResContactChunk + e - k0];
            o2 += cprod[2 * kResContactChunk + e - k0];
        }
    };
    // w = A u for the lane's row: the diagonal block, the material groups (resident ones from shared memory)
    // and the contact blocks.  Called by every thread of the block.  The rows that carry contacts sit in a
    // few slices, so the contact blocks are not walked by their rows' warps: every thread of the block
    // multiplies one block at a time (the CSR range of the block's rows, in chunks), and each row adds its
    // own products in CSR order, as the row walk would.  Lanes past n compute a discarded value.
    auto matvec = [&](float v0, float v1, float v2, float& q0, float& q1, float& q2) {
        const uint32_t first = min(ce1 - ce0, (uint32_t)kResContactChunk);
        contact_chunk(ce0, first);
        float4 c0, c1, c2;
        if (GT > 0 && ls < nsl) {  // the same in every lane of the warp
            const uint32_t db = tbase - 80u * (ls >> 2) + 400u + 12u * (ls >> 2);
            const uint4 d0 = tmem_ld4(db), d1 = tmem_ld4(db + 4u), d2 = tmem_ld4(db + 8u);
            tmem_wait_ld();
            c0 = as_f4(d0); c1 = as_f4(d1); c2 = as_f4(d2);
        } else {
            c0 = __ldg(&a.diag[3 * row]); c1 = __ldg(&a.diag[3 * row + 1]); c2 = __ldg(&a.diag[3 * row + 2]);
        }
        q0 = __fmaf_rn(c2.x, v2, __fmaf_rn(c1.x, v1, c0.x * v0));
        q1 = __fmaf_rn(c2.y, v2, __fmaf_rn(c1.y, v1, c0.y * v0));
        q2 = __fmaf_rn(c2.z, v2, __fmaf_rn(c1.z, v1, c0.z * v0));
        float o0 = 0.f, o1 = 0.f, o2 = 0.f;
        for (uint32_t g = g0; g < g1; ++g) {
            const uint32_t j = g - g0;
            const bool res = j < (uint32_t)G;
            const bool tm = !res && j < (uint32_t)(G + GT);  // the same in every lane of the warp
            const uint32_t cb = tbase + 40u * (j - (uint32_t)G);
            uint4 jc;
            if (res) {
                jc = scol[((size_t)ls * G + j) * 32 + lane];
            } else if (tm) {
                jc = tmem_ld4(cb);
                tmem_wait_ld();
            } else {
                jc = __ldg(&C4[(size_t)g * 32 + lane]);
            }
            const float4 pv[4] = {ld_u(jc.x), ld_u(jc.y), ld_u(jc.z), ld_u(jc.w)};
            const float4* vg = res ? sval + ((size_t)ls * G + j) * 9 * 32 + lane : V4 + (size_t)g * 9 * 32 + lane;
#pragma unroll
            for (int rr = 0; rr < 3; ++rr) {
                float4 ma, mb, mc;
                if (res) {
                    ma = vg[32 * rr]; mb = vg[32 * (rr + 3)]; mc = vg[32 * (rr + 6)];
                } else if (tm) {
                    const uint4 ua = tmem_ld4(cb + 4u + 4u * rr), ub = tmem_ld4(cb + 4u + 4u * (rr + 3)),
                                uc = tmem_ld4(cb + 4u + 4u * (rr + 6));
                    tmem_wait_ld();
                    ma = as_f4(ua); mb = as_f4(ub); mc = as_f4(uc);
                } else {
                    ma = ld_stream4(vg + 32 * rr); mb = ld_stream4(vg + 32 * (rr + 3)); mc = ld_stream4(vg + 32 * (rr + 6));
                }
                float o = rr == 0 ? o0 : rr == 1 ? o1 : o2;
#pragma unroll
                for (int jj = 0; jj < 4; ++jj)
                    o += __fmaf_rn(comp(mc, jj), pv[jj].z, __fmaf_rn(comp(mb, jj), pv[jj].y, comp(ma, jj) * pv[jj].x));
                if (rr == 0) o0 = o;
                else if (rr == 1) o1 = o;
                else o2 = o;
            }
        }
        if (ce1 > ce0) {
            __syncthreads();
            contact_add(ce0, first, o0, o1, o2);
            for (uint32_t k0 = ce0 + first; k0 < ce1; k0 += kResContactChunk) {  // blocks with many contacts
                const uint32_t cnt = min(ce1 - k0, (uint32_t)kResContactChunk);
                __syncthreads();
                contact_chunk(k0, cnt);
                __syncthreads();
                contact_add(k0, cnt, o0, o1, o2);
            }
        }
        q0 += o0;
        q1 += o1;
        q2 += o2;
    };
#define LCS_MINV(v0, v1, v2, o0, o1, o2)                          \
    {                                                              \
        o0 = __fmaf_rn(m6, v2, __fmaf_rn(m3, v1, m0 * v0));        \
        o1 = __fmaf_rn(m7, v2, __fmaf_rn(m4, v1, m1 * v0));        \
        o2 = __fmaf_rn(m8, v2, __fmaf_rn(m5, v1, m2 * v0));        \
    }
    float u0, u1, u2, w0 = 0.f, w1 = 0.f, w2 = 0.f;
    LCS_MINV(r0, r1, r2, u0, u1, u2)
    unsigned tag = 1u;
    if (own) __stcg(&a.pg[i], make_float4(u0, u1, u2, 0.0f));
    // a wait that ran out ends the solve (ok false in every thread of the block: the fail flag is shared);
    // the tensor memory is released on every path
    bool ok = res_publish_wait(ra.flags, tag, s_dep, a.stats, &s_fail);
    if (ok) matvec(u0, u1, u2, w0, w1, w2);  // every warp (block barrier inside)
    float x0 = 0.f, x1 = 0.f, x2 = 0.f, p0 = 0.f, p1 = 0.f, p2 = 0.f, sd0 = 0.f, sd1 = 0.f, sd2 = 0.f;
    float gamma_old = 0.0f, alpha_old = 0.0f, norm_r0 = 0.0f, norm_r = 0.0f, gamma = 0.0f;
    int iter = 0, status = 0;
    for (iter = 0; ok && iter < a.max_iter; ++iter) {
        double dg, dd, dr;
        if (a.fp64) {
            dg = (double)r0 * u0 + (double)r1 * u1 + (double)r2 * u2;
            dd = (double)w0 * u0 + (double)w1 * u1 + (double)w2 * u2;
            dr = (double)r0 * r0 + (double)r1 * r1 + (double)r2 * r2;
        } else {
            dg = __fmaf_rn(r2, u2, __fmaf_rn(r1, u1, r0 * u0));
            dd = __fmaf_rn(w2, u2, __fmaf_rn(w1, u1, w0 * u0));
            dr = __fmaf_rn(r2, r2, __fmaf_rn(r1, r1, r0 * r0));
        }
        if (!own) dg = dd = dr = 0.0;
        unsigned long long* part = reinterpret_cast<unsigned long long*>(a.part) + 4 * (size_t)P * (iter & 1);
        double sg, sdd, sr;
        if (!res_allgather3<BT>(dg, dd, dr, part, (unsigned)(iter % 15), spart, a.stats, &s_fail, sg, sdd, sr)) {
            ok = false;
            break;
        }
        gamma = (float)sg;
        const float delta = (float)sdd;
        norm_r = sqrtf((float)sr);
        if (iter == 0) norm_r0 = norm_r;
        if (iter % a.check_every == 0) {
            if (isnan(gamma) || isinf(gamma)) { status = LCS_ERR_NAN; break; }
            if (gamma < a.abs_rz_tol) break;
            if (a.rel_tol > 0.0f && norm_r <= a.rel_tol * norm_r0) break;
        }
        float beta = 0.0f, alpha = 0.0f;
        bool restart = iter == 0 || alpha_old == 0.0f;
        if (!restart) {
            beta = safe_div(gamma, gamma_old);
            const float den = delta - beta * gamma / alpha_old;
            restart = !(den >= kPcgEps);
            if (!restart) alpha = gamma / den;
        }
        if (restart) {
            beta = 0.0f;
            alpha = safe_div(gamma, delta);
        }
        p0 = u0 + beta * p0; p1 = u1 + beta * p1; p2 = u2 + beta * p2;
        sd0 = w0 + beta * sd0; sd1 = w1 + beta * sd1; sd2 = w2 + beta * sd2;
        x0 = x0 + alpha * p0; x1 = x1 + alpha * p1; x2 = x2 + alpha * p2;
        r0 -= alpha * sd0; r1 -= alpha * sd1; r2 -= alpha * sd2;
        LCS_MINV(r0, r1, r2, u0, u1, u2)
        ++tag;
        if (own) __stcg(&a.pg[i], make_float4(u0, u1, u2, 0.0f));
        if (!res_publish_wait(ra.flags, tag, s_dep, a.stats, &s_fail)) {
            ok = false;
            break;
        }
        matvec(u0, u1, u2, w0, w1, w2);
        gamma_old = gamma;
        alpha_old = alpha;
    }
#undef LCS_MINV
    if (ok) {
        if (own) a.x[i] = make_float4(x0, x1, x2, 0.0f);
        if (c == 0 && t == 0) {
            a.stats->iterations = iter;
            a.stats->rel_residual = norm_r0 > 0.0f ? norm_r / norm_r0 : 0.0f;
            a.stats->dot_rz = gamma;
            if (a.stats->status == LCS_OK) a.stats->status = status;
        }
    }
    if (GT > 0) {  // every warp's tensor-memory reads are complete (each waited for them)
        tmem_fence_before();
        __syncthreads();
        if (ls == 0) tmem_dealloc(s_taddr, kResTmemCols);
    }
}

// ------------------------------------------------------------------------ batched scenes
// Many independent systems (one per scene, rows [roff[s], roff[s+1])) solved in one launch: one
// thread-block cluster per scene, synchronised by the hardware cluster barrier, with the scene's
// own alpha, beta and stop decision (the recurrences and stop rules of k_pcg_fused).  The rows of a
// scene are cut into chunks of 256; chunk k belongs to CTA k mod C of the cluster, thread t to row
// 256k + t (the SpMV uses 4 lanes per row).  Every dot product is summed per chunk in a fixed tree
// and then over the chunks in a fixed order, so a scene's result does not depend on the cluster
// size C nor on the other scenes of the launch.  Vectors live in global memory (L2-resident per
// scene); cross-CTA reads use ld.cg.
constexpr int kBatchThreads = 256;
constexpr int kBatchLanes = 4;

struct BatchArgs {
    const uint32_t* scenes;  // cluster index -> scene id (null: the identity)
    const uint32_t* roff;    // S + 1
    const uint32_t* active;  // S (0: skip the scene, x = 0) or null
    const float4* diag;
    Bsr A, B;
    const float4* b;
    float4* x;
    float4 *r, *z, *p, *q, *minv;
    double* cpart;           // 4 doubles per chunk; chunk k of scene s at (roff[s] >> 8) + s + k
    int max_iter;
    float rel_tol, abs_rz_tol;
    int check_every;
    int fp64;
    lcs_pcg_stats* stats;    // S
};

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t cluster_ctas()
{
    uint32_t n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return n;
}

// fixed-tree sum of one value per thread (256 threads) -> thread 0
__device__ __forceinline__ double chunk_sum(double v, double* s_w)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane_id() == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
#pragma unroll
        for (int w = 0; w < kBatchThreads / 32; ++w) t += s_w[w];
    __syncthreads();
    return t;
}

// sum over a scene's chunks in a fixed order, the same in every CTA of the cluster
__device__ __forceinline__ void scene_sum(const double* cp, uint32_t nchunks, int k, int count, double* out,
                                          double* s_out)
{
    if (threadIdx.x < 32) {
        double v[2] = {0.0, 0.0};
        for (uint32_t c = threadIdx.x; c < nchunks; c += 32)
            for (int j = 0; j < count; ++j) v[j] += __ldcg(&cp[4 * c + k + j]);
        for (int j = 0; j < count; ++j) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xFFFFFFFFu, v[j], o);
        }
        if (threadIdx.x == 0)
            for (int j = 0; j < count; ++j) s_out[j] = v[j];
    }
    __syncthreads();
    for (int j = 0; j < count; ++j) out[j] = s_out[j];
    __syncthreads();
}

__global__ void __launch_bounds__(kBatchThreads) k_pcg_batch(BatchArgs a)
{
    __shared__ double s_w[kBatchThreads / 32];
    __shared__ double s_out[2];
    __shared__ double s_pq[kBatchThreads];
    const uint32_t C = cluster_ctas(), rank = cluster_rank();
    const uint32_t s = a.scenes ? a.scenes[blockIdx.x / C] : blockIdx.x / C;
    const uint32_t r0 = a.roff[s], r1 = a.roff[s + 1], nrows = r1 - r0;
    const uint32_t nchunks = (nrows + kBatchThreads - 1) / kBatchThreads;
    double* cp = a.cpart + 4 * (size_t)((r0 >> 8) + s);
    const uint32_t t = threadIdx.x;
    const bool on = !a.active || a.active[s] != 0u;  // uniform over the cluster
    for (uint32_t k = rank; k < nchunks; k += C) {
        const uint32_t i = r0 + k * kBatchThreads + t;
        if (i >= r1) continue;
        a.x[i] = make_float4(0, 0, 0, 0);
        if (!on) continue;
        a.r[i] = a.b[i];
        a.p[i] = make_float4(0, 0, 0, 0);
        const float4 c0 = a.diag[3 * i], c1 = a.diag[3 * i + 1], c2 = a.diag[3 * i + 2];
        const float aa = c0.x, bb = c1.x, c = c2.x, d = c0.y, e = c1.y, f = c2.y, g = c0.z, h = c1.z, kk = c2.z;
        const float A = e * kk - f * h, B = f * g - d * kk, Cc = d * h - e * g;
        const float id = 1.0f / (aa * A + bb * B + c * Cc);
        a.minv[3 * i + 0] = make_float4(A * id, B * id, Cc * id, 0.0f);
        a.minv[3 * i + 1] = make_float4((c * h - bb * kk) * id, (aa * kk - c * g) * id, (bb * g - aa * h) * id, 0.0f);
        a.minv[3 * i + 2] = make_float4((bb * f - c * e) * id, (c * d - aa * f) * id, (aa * e - bb * d) * id, 0.0f);
    }
    if (!on) {
        if (rank == 0 && t == 0) a.stats[s] = lcs_pcg_stats{0, 0.0f, 0.0f, LCS_OK};
        return;
    }
    float rz_old = 0.0f, norm_r0 = 0.0f, norm_r = 0.0f, rz = 0.0f;
    int iter = 0, status = 0;
    for (iter = 0; iter < a.max_iter; ++iter) {
        // z = Minv r ; r.r ; r.z per chunk
        for (uint32_t k = rank; k < nchunks; k += C) {
            const uint32_t i = r0 + k * kBatchThreads + t;
            double drr = 0.0, drz = 0.0;
            if (i < r1) {
                const float4 rv = a.r[i];
                const float3 zv = mv12(a.minv + 3 * (size_t)i, rv);
                a.z[i] = make_float4(zv.x, zv.y, zv.z, 0.0f);
                if (a.fp64) {
                    drr = (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z;
                    drz = (double)rv.x * zv.x + (double)rv.y * zv.y + (double)rv.z * zv.z;
                } else {
                    drr = __fmaf_rn(rv.z, rv.z, __fmaf_rn(rv.y, rv.y, rv.x * rv.x));
                    drz = __fmaf_rn(rv.z, zv.z, __fmaf_rn(rv.y, zv.y, rv.x * zv.x));
                }
            }
            const double srr = chunk_sum(drr, s_w), srz = chunk_sum(drz, s_w);
            if (t == 0) {
                cp[4 * k + 0] = srr;
                cp[4 * k + 1] = srz;
            }
        }
        cluster_sync_all();
        double red[2];
        scene_sum(cp, nchunks, 0, 2, red, s_out);
        const float rr = (float)red[0];
        rz = (float)red[1];
        const float beta = safe_div(rz, rz_old);
        rz_old = rz;
        norm_r = sqrtf(rr);
        if (iter == 0) norm_r0 = norm_r;
        if (iter % a.check_every == 0) {
            if (isnan(rz) || isinf(rz)) { status = LCS_ERR_NAN; break; }
            if (rz < a.abs_rz_tol) break;
            if (a.rel_tol > 0.0f && norm_r <= a.rel_tol * norm_r0) break;
        }
        for (uint32_t k = rank; k < nchunks; k += C) {
            const uint32_t i = r0 + k * kBatchThreads + t;
            if (i < r1) {
                const float4 zv = a.z[i], pv = a.p[i];
                a.p[i] = make_float4(zv.x + beta * pv.x, zv.y + beta * pv.y, zv.z + beta * pv.z, 0.0f);
            }
        }
        cluster_sync_all();
        // q = A p (4 lanes per row) ; p.q per chunk
        for (uint32_t k = rank; k < nchunks; k += C) {
            const uint32_t base = r0 + k * kBatchThreads;
            const uint32_t lig = t % kBatchLanes;
            for (uint32_t rr_ = t / kBatchLanes; rr_ < (uint32_t)kBatchThreads; rr_ += kBatchThreads / kBatchLanes) {
                const uint32_t row = base + rr_ < r1 ? base + rr_ : r1 - 1;  // whole groups stay converged
                const float3 qv = row_product<kBatchLanes>(row, lig, a.diag, a.A, a.B, a.p);
                if (lig == 0) {
                    double d = 0.0;
                    if (base + rr_ < r1) {
                        a.q[row] = make_float4(qv.x, qv.y, qv.z, 0.0f);
                        const float4 pv = __ldcg(&a.p[row]);
                        d = a.fp64 ? (double)pv.x * qv.x + (double)pv.y * qv.y + (double)pv.z * qv.z
                                   : (double)__fmaf_rn(pv.z, qv.z, __fmaf_rn(pv.y, qv.y, pv.x * qv.x));
                    }
                    s_pq[rr_] = d;
                }
            }
            __syncthreads();
            const double spq = chunk_sum(s_pq[t], s_w);
            if (t == 0) cp[4 * k + 2] = spq;
        }
        cluster_sync_all();
        double pq;
        scene_sum(cp, nchunks, 2, 1, &pq, s_out);
        const float alpha = safe_div(rz, (float)pq);
        for (uint32_t k = rank; k < nchunks; k += C) {
            const uint32_t i = r0 + k * kBatchThreads + t;
            if (i < r1) {
                const float4 pv = a.p[i], qv = __ldcg(&a.q[i]), xv = a.x[i], rv = a.r[i];
                a.x[i] = make_float4(xv.x + alpha * pv.x, xv.y + alpha * pv.y, xv.z + alpha * pv.z, 0.0f);
                a.r[i] = make_float4(rv.x - alpha * qv.x, rv.y - alpha * qv.y, rv.z - alpha * qv.z, 0.0f);
            }
        }
    }
    if (rank == 0 && t == 0) {
        lcs_pcg_stats st;
        st.iterations = iter;
        st.rel_residual = norm_r0 > 0.0f ? norm_r / norm_r0 : 0.0f;
        st.dot_rz = rz_old;
        st.status = status;
        a.stats[s] = st;
    }
}

}  // namespace

// a CSR matrix rewritten as SELL-32 (4-slot groups): per-slice widths and slot offsets, columns, values
struct SellBuf {
    uint32_t *width = nullptr, *ptr = nullptr, *col = nullptr;
    float* val = nullptr;
    int* ok = nullptr;
    uint32_t cap = 0;  // slots the buffers hold
};

struct lcs_pcg {
    uint32_t n = 0;
    float4 *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *minv = nullptr;
    double* part = nullptr;
    float* part_f = nullptr;
    float* scal = nullptr;       // plain-mode scalars
    float* h_scal = nullptr;     // pinned host copy
    unsigned* bar = nullptr;     // [count, gen]
    unsigned* flags = nullptr;   // slice-resident solve: per-block publication tags (kResMaxBlocks)
    int res_gres = -2;           // slice-resident solve: resident groups per slice (-2: not set up)
    uint32_t res_blocks = 0, res_slices = 0, res_max_slices = 0;
    uint32_t *res_part = nullptr, *res_owner = nullptr;  // slice partition (per solve)
    size_t res_smem = 0;
    uint32_t tuned_target = 0;   // batched solves: chunks of 256 rows per CTA picking each scene's cluster (0: untuned)
    float tuned_ms = 0.0f;       // the tuned configuration's solve time
    lcs_pcg_stats* d_stats = nullptr;
    int fused_grid = 0;
    int rows_capacity = -1;  // most rows the row-resident solve can hold co-resident (-1: not queried)
    double* cpart = nullptr;  // batched solve: per-chunk partial sums
    size_t cpart_cap = 0;     // chunks
    // batched solve with per-scene cluster sizes: scene lists per size class, one stream per class
    uint32_t* class_scenes = nullptr;
    size_t class_cap = 0;
    std::vector<uint32_t> class_host;
    cudaStream_t class_stream[5] = {};
    cudaEvent_t class_fork = nullptr, class_join[5] = {};
    // the CSR material and contact matrices of lcs_pcg_solve rewritten as SELL-32 for the row-resident solves
    SellBuf msell, csell;
};

static constexpr int kRowLanes = 4;
static constexpr int kPlainBlocks = 256;
static constexpr int kRowMaxBlocks = 1024;
static constexpr int kPcgNoResident = LCS_PCG_INTERNAL_NO_RESIDENT;

extern "C" int lcs_debug_pcg_wait(int32_t which, int32_t missing_block, uint32_t blocks, uint32_t spin_limit,
                                  lcs_stream stream)
{
    if (which != 0 && which != 1) return lcs_fail(LCS_ERR_INVALID, "lcs_debug_pcg_wait: which must be 0 or 1");
    if (blocks < 2 || blocks > 32 || blocks > (uint32_t)kResMaxBlocks)
        return lcs_fail(LCS_ERR_INVALID, "lcs_debug_pcg_wait: blocks must be in [2, 32]");
    if (spin_limit == 0 || spin_limit > kBarrierSpinLimit)
        return lcs_fail(LCS_ERR_INVALID, "lcs_debug_pcg_wait: spin_limit must be in [1, 2^24]");
    if (missing_block >= (int32_t)blocks) return lcs_fail(LCS_ERR_INVALID, "lcs_debug_pcg_wait: no such block");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned* words = nullptr;  // tagged partials (8 words per block), flags (kResFlagStride per block)
    lcs_pcg_stats* st = nullptr;
    const size_t n_words = 8 * (size_t)blocks + (size_t)kResFlagStride * blocks;
    LCS_CUDA_TRY(cudaMalloc(&words, 4 * n_words));
    if (cudaMalloc(&st, sizeof(lcs_pcg_stats)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(words);
        return lcs_fail(LCS_ERR_CUDA, "lcs_debug_pcg_wait: cudaMalloc failed");
    }
    lcs_pcg_stats h{};
    int rc = LCS_OK;
    if (cudaMemsetAsync(words, 0xFF, 32 * (size_t)blocks, s) != cudaSuccess ||
        cudaMemsetAsync(words + 8 * (size_t)blocks, 0, 4 * (size_t)kResFlagStride * blocks, s) != cudaSuccess ||
        cudaMemsetAsync(st, 0, sizeof(h), s) != cudaSuccess)
        rc = LCS_ERR_CUDA;
    unsigned long long* part = reinterpret_cast<unsigned long long*>(words);
    unsigned* flags = words + 8 * (size_t)blocks;
    void* args[] = {&which, &missing_block, &spin_limit, &part, &flags, &st};
    if (rc == LCS_OK &&
        cudaLaunchCooperativeKernel((const void*)k_wait_probe, dim3(blocks), dim3(128), args, 0, s) != cudaSuccess)
        rc = LCS_ERR_CUDA;
    if (rc == LCS_OK) lcs_count_launch();
    if (rc == LCS_OK && (cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess))
        rc = LCS_ERR_CUDA;
    const cudaError_t err = cudaGetLastError();
    cudaFree(words);
    cudaFree(st);
    if (rc != LCS_OK) return lcs_fail(rc, cudaGetErrorString(err));
    if (h.status == LCS_ERR_TIMEOUT)
        return lcs_fail(LCS_ERR_TIMEOUT, "lcs_debug_pcg_wait: a bounded wait ran out (LCS_ERR_TIMEOUT)");
    return h.status;
}

extern "C" int lcs_pcg_create(uint32_t n, lcs_pcg** out)
{
    if (!out || n == 0) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_create: bad argument");
    lcs_pcg* p = new (std::nothrow) lcs_pcg();
    if (!p) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_create: out of host memory");
    p->n = n;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_fused<kRowLanes>, kFusedThreads, 0);
    if (per_sm > 1) per_sm = 1;
    p->fused_grid = sms * (per_sm > 0 ? per_sm : 1);
    // fused: 3 doubles per block; row-resident: 4 per block, twice (alternate iterations) for up to kRowMaxBlocks
    const int parts = 8 * kRowMaxBlocks / 3 + 1 + (p->fused_grid > kPlainBlocks ? p->fused_grid : kPlainBlocks);
    cudaError_t e = cudaSuccess;
    auto A = [&](void** q, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(q, bytes); };
    A((void**)&p->r, 16 * (size_t)n);
    A((void**)&p->z, 16 * (size_t)n);
    A((void**)&p->p, 16 * (size_t)n);
    A((void**)&p->q, 16 * (size_t)n);
    A((void**)&p->minv, 48 * (size_t)n);
    A((void**)&p->part, 3 * sizeof(double) * parts);
    A((void**)&p->part_f, 3 * sizeof(float) * parts);
    A((void**)&p->scal, 16 * sizeof(float));
    A((void**)&p->bar, 2 * sizeof(unsigned));
    A((void**)&p->flags, kResFlagStride * kResMaxBlocks * sizeof(unsigned));
    A((void**)&p->d_stats, sizeof(lcs_pcg_stats));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&p->h_scal, 16 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(p->bar, 0, 2 * sizeof(unsigned));
    if (e != cudaSuccess) {
        lcs_pcg_destroy(p);
        return lcs_fail(LCS_ERR_CUDA, "lcs_pcg_create: allocation failed");
    }
    *out = p;
    return LCS_OK;
}

extern "C" int lcs_pcg_destroy(lcs_pcg* p)
{
    if (!p) return LCS_OK;
    void* ptrs[] = {p->r, p->z, p->p, p->q, p->minv, p->part, p->part_f, p->scal, p->bar, p->flags, p->d_stats,
                    p->cpart, p->class_scenes, p->res_part, p->res_owner, p->msell.width, p->msell.ptr,
                    p->msell.col, p->msell.val, p->msell.ok, p->csell.width, p->csell.ptr, p->csell.col,
                    p->csell.val, p->csell.ok};
    for (int k = 0; k < 5; ++k) {
        if (p->class_stream[k]) {
            cudaStreamSynchronize(p->class_stream[k]);
            cudaStreamDestroy(p->class_stream[k]);
        }
        if (p->class_join[k]) cudaEventDestroy(p->class_join[k]);
    }
    if (p->class_fork) cudaEventDestroy(p->class_fork);
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (p->h_scal) cudaFreeHost(p->h_scal);
    delete p;
    return LCS_OK;
}

extern "C" const lcs_pcg_stats* lcs_pcg_device_stats(const lcs_pcg* p) { return p ? p->d_stats : nullptr; }

static Bsr to_bsr(const lcs_bsr* m) { return m ? Bsr{m->row_ptr, m->col, m->val} : Bsr{nullptr, nullptr, nullptr}; }

extern "C" int lcs_spmv(uint32_t n, const float* diag, const lcs_bsr* A, const lcs_bsr* B, const float* x, float* y,
                        lcs_stream stream)
{
    if (!diag || !x || !y || n == 0) return lcs_fail(LCS_ERR_INVALID, "lcs_spmv: bad argument");
    if ((A && A->n_rows != n) || (B && B->n_rows != n)) return lcs_fail(LCS_ERR_INVALID, "lcs_spmv: row count mismatch");
    k_spmv<kRowLanes><<<grid_for((uint64_t)n * kRowLanes, 256), 256, 0, (cudaStream_t)stream>>>(
        n, reinterpret_cast<const float4*>(diag), to_bsr(A), to_bsr(B), reinterpret_cast<const float4*>(x),
        reinterpret_cast<float4*>(y));
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

template <typename T>
static int plain_solve(lcs_pcg* P, const float4* diag, Bsr A, Bsr B, const float4* b, float4* x,
                       const lcs_pcg_opts& o, lcs_pcg_stats* stats, cudaStream_t s)
{
    const uint32_t n = P->n;
    const int g = grid_for(n, 256);
    const int nb = g < kPlainBlocks ? g : kPlainBlocks;
    T* part = reinterpret_cast<T*>(sizeof(T) == 8 ? (void*)P->part : (void*)P->part_f);
    k_plain_init<<<g, 256, 0, s>>>(n, b, diag, x, P->r, P->p, P->minv, P->scal);
    lcs_count_launch();
    int iter = 0, status = LCS_OK;
    float norm_r0 = 0.0f, norm_r = 0.0f, rz = 0.0f;
    const int check = o.check_every > 0 ? o.check_every : 1;
    for (iter = 0; iter < o.max_iter; ++iter) {
        k_plain_precond<T><<<nb, 256, 0, s>>>(n, P->minv, P->r, P->z, part);
        lcs_count_launch();
        k_plain_precond2<T><<<1, 256, 0, s>>>(part, nb, P->scal, iter == 0);
        lcs_count_launch();
        if (iter % check == 0) {
            LCS_CUDA_TRY(cudaMemcpyAsync(P->h_scal, P->scal, 8 * sizeof(float), cudaMemcpyDeviceToHost, s));
            LCS_CUDA_TRY(cudaStreamSynchronize(s));
            rz = P->h_scal[1];
            norm_r = P->h_scal[4];
            if (iter == 0) norm_r0 = norm_r;
            if (isnan(rz) || isinf(rz)) { status = LCS_ERR_NAN; break; }
            if (rz < o.abs_rz_tol) break;
            if (o.rel_tol > 0.0f && norm_r <= o.rel_tol * norm_r0) break;
        }
        k_plain_update_p<<<g, 256, 0, s>>>(n, P->z, P->p, P->scal);
        lcs_count_launch();
        k_spmv<kRowLanes><<<grid_for((uint64_t)n * kRowLanes, 256), 256, 0, s>>>(n, diag, A, B, P->p, P->q);
        lcs_count_launch();
        k_plain_dot<T><<<nb, 256, 0, s>>>(n, P->p, P->q, part);
        lcs_count_launch();
        k_plain_alpha<T><<<1, 256, 0, s>>>(part, nb, P->scal);
        lcs_count_launch();
        k_plain_step<<<g, 256, 0, s>>>(n, x, P->r, P->p, P->q, P->scal);
        lcs_count_launch();
    }
    LCS_LAUNCH_CHECK();
    LCS_CUDA_TRY(cudaMemcpyAsync(P->h_scal, P->scal, 8 * sizeof(float), cudaMemcpyDeviceToHost, s));
    LCS_CUDA_TRY(cudaStreamSynchronize(s));
    lcs_pcg_stats local;
    local.iterations = iter;
    local.rel_residual = norm_r0 > 0.0f ? P->h_scal[4] / norm_r0 : 0.0f;
    local.dot_rz = P->h_scal[1];
    local.status = status;
    if (stats) *stats = local;
    // keep the device copy of the stats current too (pageable source: staged before return)
    LCS_CUDA_TRY(cudaMemcpyAsync(P->d_stats, &local, sizeof(local), cudaMemcpyHostToDevice, s));
    return status == LCS_OK ? LCS_OK : lcs_fail(status, "lcs_pcg_solve: NaN/Inf in r.z");
}

// Launch shape of the slice-resident solve for P->n rows: one block per SM (fewer when there are fewer
// slices), at most kResThreads / 32 slices per block, and as many resident groups per slice as the
// shared memory left after u and the partial sums holds.  LCS_ERR_CAPACITY when it does not apply.
static int res_setup(lcs_pcg* P)
{
    if (P->res_gres >= 0) return LCS_OK;
    if (P->res_gres == -1) return LCS_ERR_CAPACITY;
    P->res_gres = -1;
    int dev = 0, sms = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LCS_ERR_CAPACITY;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const uint32_t S = (P->n + 31) / 32;
    uint32_t blocks = (uint32_t)sms < S ? (uint32_t)sms : S;
    if (blocks > (uint32_t)kResMaxBlocks) blocks = kResMaxBlocks;
    if (blocks > (uint32_t)kResThreads) blocks = kResThreads;  // one waiting thread per block
    if (blocks == 0) return LCS_ERR_CAPACITY;
    if ((S + blocks - 1) / blocks > (uint32_t)(kResThreads / 32)) return LCS_ERR_CAPACITY;
    // room for a full block of slices, so that the per-solve partition can balance cost
    const uint32_t max_slices = S < (uint32_t)(kResThreads / 32) ? S : (uint32_t)(kResThreads / 32);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_pcg_res<kResThreads>) != cudaSuccess) return LCS_ERR_CAPACITY;
    const size_t base = sizeof(float) * 3 * kResContactChunk + 32 * (size_t)blocks;
    const size_t avail = (size_t)optin > fa.sharedSizeBytes + base ? (size_t)optin - fa.sharedSizeBytes - base : 0;
    size_t gres = avail / ((size_t)max_slices * kResGroupBytes);
    if (gres > 8) gres = 8;
    const size_t dyn = base + gres * max_slices * kResGroupBytes;
    if (cudaFuncSetAttribute(k_pcg_res<kResThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) !=
        cudaSuccess) {
        cudaGetLastError();
        return LCS_ERR_CAPACITY;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_res<kResThreads>, kResThreads, dyn);
    if (per_sm < 1 || (int64_t)per_sm * sms < (int64_t)blocks) return LCS_ERR_CAPACITY;
    if (cudaMalloc((void**)&P->res_part, sizeof(uint32_t) * (blocks + 1)) != cudaSuccess ||
        cudaMalloc((void**)&P->res_owner, sizeof(uint32_t) * S) != cudaSuccess) {
        cudaGetLastError();
        return LCS_ERR_CAPACITY;
    }
    P->res_blocks = blocks;
    P->res_slices = S;
    P->res_max_slices = max_slices;
    P->res_smem = dyn;
    P->res_gres = (int)gres;
    return LCS_OK;
}

// ------------------------------------------------ contact blocks as SELL-32 (once per Newton iteration)
// The contact CSR rewritten in the material matrix's SELL-32 layout, so that the row-resident solves
// read a row's contact blocks like its material blocks: coalesced 16-B loads, slot order = CSR order
// (the same sums as the CSR walk).  k_csell_width: slots per slice (the slice's longest row, rounded up
// to 4); k_csell_scan: slice offsets and the fit flag; k_csell_fill: columns and values at their SELL
// positions, padding slots as zero blocks against the row itself.
__global__ void k_csell_width(uint32_t n, const uint32_t* __restrict__ rp, uint32_t* __restrict__ width)
{
    const uint32_t S = (n + 31) / 32, lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < S; s += warps) {
        const uint32_t r = 32 * s + lane;
        const uint32_t len = r < n ? __ldcg(&rp[r + 1]) - __ldcg(&rp[r]) : 0u;
        const uint32_t w = __reduce_max_sync(0xFFFFFFFFu, len);
        if (lane == 0) width[s] = (w + 3u) & ~3u;
    }
}

__global__ void __launch_bounds__(1024) k_csell_scan(uint32_t S, const uint32_t* __restrict__ width,
                                                     uint32_t* __restrict__ ptr, uint32_t cap_slots, int* ok)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t carry;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    if (t == 0) carry = 0u;
    __syncthreads();
    for (uint32_t base = 0; base < S; base += 1024u) {
        const uint32_t s = base + t;
        const uint32_t v = s < S ? width[s] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += x;
        }
        if (lane == 31u) ws[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = ws[lane];
#pragma unroll
            for (uint32_t o = 1; o < 32u; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= o) w += x;
            }
            ws[lane] = w;
        }
        __syncthreads();
        const uint32_t pre = carry + (warp ? ws[warp - 1] : 0u);
        if (s < S) ptr[s] = pre + incl - v;
        __syncthreads();
        if (t == 0) carry += ws[31];
        __syncthreads();
    }
    if (t == 0) {
        ptr[S] = carry;
        *ok = carry <= cap_slots ? 1 : 0;
    }
}

__global__ void k_csell_fill(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col,
                             const float* __restrict__ val, const uint32_t* __restrict__ ptr, const int* __restrict__ ok,
                             uint32_t* __restrict__ scol, float* __restrict__ sval)
{
    if (!*ok) return;
    const uint32_t rows = 32u * ((n + 31) / 32);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const uint32_t s = r >> 5, lane = r & 31u;
        const uint32_t p0 = ptr[s], w = ptr[s + 1] - p0;
        const uint32_t k0 = r < n ? rp[r] : 0u, len = r < n ? rp[r + 1] - k0 : 0u;
        const uint32_t pad = r < n ? r : n - 1;
        for (uint32_t j = 0; j < w; ++j) {
            const size_t slot = (size_t)p0 + j, g = slot >> 2, jj = slot & 3u;
            const bool real = j < len;
            scol[(g * 32 + lane) * 4 + jj] = real ? col[k0 + j] : pad;
#pragma unroll
            for (int c = 0; c < 9; ++c)
                sval[((g * 9 + c) * 32 + lane) * 4 + jj] = real ? val[9 * ((size_t)k0 + j) + c] : 0.0f;
        }
    }
}

int lcs_contact_to_sell(uint32_t n, const lcs_bsr* B, uint32_t* width, uint32_t* ptr, uint32_t* col, float* val,
                        uint32_t cap_slots, int* ok, lcs_stream stream)
{
    if (!B || !B->row_ptr || !width || !ptr || !col || !val || !ok || n == 0)
        return lcs_fail(LCS_ERR_INVALID, "lcs_contact_to_sell: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t S = (n + 31) / 32;
    k_csell_width<<<grid_for((uint64_t)S * 32, 256), 256, 0, s>>>(n, B->row_ptr, width);
    k_csell_scan<<<1, 1024, 0, s>>>(S, width, ptr, cap_slots, ok);
    k_csell_fill<<<grid_for((uint64_t)S * 32, 256), 256, 0, s>>>(n, B->row_ptr, B->col, B->val, ptr, ok, col, val);
    for (int k = 0; k < 3; ++k) lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

int lcs_pcg_resident(lcs_pcg* P) { return P && res_setup(P) == LCS_OK ? 1 : 0; }

// A CSR matrix of lcs_pcg_solve as SELL-32, the layout the Newton loop's producers write: slot order is
// CSR order, so each row's block products are summed in the order of the CSR walk.  The padded slot count
// is read back once per call; the buffers grow when it exceeds the last call's.
static int csr_to_sell(SellBuf& sb, uint32_t n, const lcs_bsr* M, cudaStream_t s)
{
    const uint32_t S = (n + 31) / 32;
    if (!sb.width) {
        if (cudaMalloc((void**)&sb.width, sizeof(uint32_t) * S) != cudaSuccess ||
            cudaMalloc((void**)&sb.ptr, sizeof(uint32_t) * (S + 1)) != cudaSuccess ||
            cudaMalloc((void**)&sb.ok, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return lcs_fail(LCS_ERR_CUDA, "lcs_pcg_solve: SELL-32 buffers: allocation failed");
        }
    }
    k_csell_width<<<grid_for((uint64_t)S * 32, 256), 256, 0, s>>>(n, M->row_ptr, sb.width);
    k_csell_scan<<<1, 1024, 0, s>>>(S, sb.width, sb.ptr, sb.cap, sb.ok);
    lcs_count_launch();
    lcs_count_launch();
    uint32_t slots = 0;
    LCS_CUDA_TRY(cudaMemcpyAsync(&slots, sb.ptr + S, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    LCS_CUDA_TRY(cudaStreamSynchronize(s));
    if (slots > sb.cap) {
        if (sb.col) cudaFree(sb.col);
        if (sb.val) cudaFree(sb.val);
        sb.col = nullptr;
        sb.val = nullptr;
        sb.cap = 0;
        const uint32_t cap = slots + slots / 8 + 128;
        if (cudaMalloc((void**)&sb.col, sizeof(uint32_t) * 32 * (size_t)cap) != cudaSuccess ||
            cudaMalloc((void**)&sb.val, sizeof(float) * 9 * 32 * (size_t)cap) != cudaSuccess) {
            cudaGetLastError();
            return lcs_fail(LCS_ERR_CUDA, "lcs_pcg_solve: SELL-32 buffers: allocation failed");
        }
        sb.cap = cap;
        k_csell_scan<<<1, 1024, 0, s>>>(S, sb.width, sb.ptr, sb.cap, sb.ok);
        lcs_count_launch();
    }
    k_csell_fill<<<grid_for((uint64_t)S * 32, 256), 256, 0, s>>>(n, M->row_ptr, M->col, M->val, sb.ptr, sb.ok, sb.col,
                                                                  sb.val);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

// row-resident solve; LCS_ERR_CAPACITY when one thread per row does not fit co-resident
static int rows_solve(lcs_pcg* P, const float4* diag, int sell, const uint32_t* m_ptr, const uint32_t* m_col,
                      const float* m_val, Bsr B, const float4* b, float4* x, const lcs_pcg_opts& o,
                      lcs_pcg_stats* stats, cudaStream_t s, const uint32_t* c_ptr = nullptr,
                      const uint32_t* c_col = nullptr, const float* c_val = nullptr, const int* c_ok = nullptr)
{
    if (P->rows_capacity < 0) P->rows_capacity = (int)lcs_pcg_rows_capacity();
    if ((int64_t)P->n > P->rows_capacity) return LCS_ERR_CAPACITY;
    const bool pipe = (o.flags & LCS_PCG_SINGLE_REDUCTION) != 0;
    if (pipe && (P->n + kRowThreads - 1) / kRowThreads > (uint32_t)kPipeMaxBlocks) return LCS_ERR_CAPACITY;
    RowArgs a;
    a.n = P->n;
    a.diag = diag;
    a.sell = sell;
    a.m_ptr = m_ptr;
    a.m_col = m_col;
    a.m_val = m_val;
    a.B = B;
    a.b_vec = B.val && (reinterpret_cast<uintptr_t>(B.val) & 15u) == 0;
    const bool cs = sell && c_ptr && c_col && c_val && c_ok;
    a.c_ptr = cs ? c_ptr : nullptr;
    a.c_col = cs ? c_col : nullptr;
    a.c_val = cs ? c_val : nullptr;
    a.c_ok = cs ? c_ok : nullptr;
    a.b = b;
    a.x = x;
    a.pg = P->p;
    a.part = P->part;
    a.bar_count = P->bar;
    a.bar_gen = P->bar + 1;
    a.max_iter = o.max_iter;
    a.rel_tol = o.rel_tol;
    a.abs_rz_tol = o.abs_rz_tol;
    a.check_every = o.check_every;
    a.fp64 = (o.flags & LCS_PCG_FP64_DOTS) ? 1 : 0;
    a.stats = P->d_stats;
    LCS_CUDA_TRY(cudaMemsetAsync(P->d_stats, 0, sizeof(lcs_pcg_stats), s));
    LCS_CUDA_TRY(cudaMemsetAsync(P->bar, 0, sizeof(unsigned), s));
    void* args[] = {&a};
    const int grid = (int)((P->n + kRowThreads - 1) / kRowThreads);
    if (pipe && sell && !(o.flags & kPcgNoResident) && res_setup(P) == LCS_OK) {
        k_res_partition<<<1, 1024, 0, s>>>(P->res_slices, P->res_blocks, P->res_max_slices, m_ptr, a.B.rp, P->n,
                                           P->res_part, P->res_owner, (uint32_t)P->res_gres);
        lcs_count_launch();
        ResArgs ra{a, P->res_part, P->res_owner, P->flags, P->res_slices, P->res_max_slices, P->res_gres,
                   kResTmemGroups};
        void* rargs[] = {&ra};
        LCS_CUDA_TRY(cudaMemsetAsync(P->flags, 0, sizeof(unsigned) * kResFlagStride * P->res_blocks, s));
        LCS_CUDA_TRY(cudaMemsetAsync(P->part, 0xFF, sizeof(double) * 8 * P->res_blocks, s));  // empty slots
        LCS_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_pcg_res<kResThreads>, dim3(P->res_blocks),
                                                 dim3(kResThreads), rargs, P->res_smem, s));
    } else if (pipe)
        LCS_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_pcg_cg1<kRowThreads>, dim3(grid), dim3(kRowThreads),
                                                 args, 0, s));
    else
        LCS_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_pcg_rows<kRowThreads>, dim3(grid), dim3(kRowThreads),
                                                 args, 0, s));
    lcs_count_launch();
    if (stats && !(o.flags & LCS_PCG_NO_STATS)) {
        LCS_CUDA_TRY(cudaMemcpyAsync(stats, P->d_stats, sizeof(lcs_pcg_stats), cudaMemcpyDeviceToHost, s));
        LCS_CUDA_TRY(cudaStreamSynchronize(s));
        if (stats->status != LCS_OK) return lcs_fail(stats->status, "lcs_pcg_solve: row-resident solve failed");
    }
    return LCS_OK;
}

// rows both row-resident kernels hold co-resident (the smaller of their occupancies)
int64_t lcs_pcg_rows_capacity()
{
    int dev = 0, sms = 0, per_sm = 0, per_sm2 = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_rows<kRowThreads>, kRowThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_pcg_cg1<kRowThreads>, kRowThreads, 0);
    if (per_sm2 < per_sm) per_sm = per_sm2;
    int64_t blocks = (int64_t)sms * per_sm;
    if (blocks > kRowMaxBlocks) blocks = kRowMaxBlocks;  // partial-sum space
    return blocks * kRowThreads;
}

int lcs_pcg_solve_sell(lcs_pcg* P, const float* diag, const uint32_t* slice_ptr, const uint32_t* col,
                       const float* val, const lcs_bsr* B, const float* b, float* x, const lcs_pcg_opts* opts,
                       lcs_pcg_stats* stats, lcs_stream stream, const uint32_t* c_ptr, const uint32_t* c_col,
                       const float* c_val, const int* c_ok)
{
    if (!P || !diag || !b || !x || !opts) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_sell: bad argument");
    return rows_solve(P, reinterpret_cast<const float4*>(diag), 1, slice_ptr, col, val, to_bsr(B),
                      reinterpret_cast<const float4*>(b), reinterpret_cast<float4*>(x), *opts, stats,
                      (cudaStream_t)stream, c_ptr, c_col, c_val, c_ok);
}

extern "C" int lcs_pcg_solve(lcs_pcg* P, const float* diag, const lcs_bsr* A, const lcs_bsr* B, const float* b,
                             float* x, const lcs_pcg_opts* opts, lcs_pcg_stats* stats, lcs_stream stream)
{
    if (!P || !diag || !b || !x) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve: bad argument");
    if ((A && A->n_rows != P->n) || (B && B->n_rows != P->n)) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve: row count mismatch");
    lcs_pcg_opts o = opts ? *opts : lcs_pcg_opts{100, 1e-4f, 1e-10f, 25, 0};
    if (o.check_every <= 0) o.check_every = 1;
    cudaStream_t s = (cudaStream_t)stream;
    const float4* d4 = reinterpret_cast<const float4*>(diag);
    const float4* b4 = reinterpret_cast<const float4*>(b);
    float4* x4 = reinterpret_cast<float4*>(x);
    if ((o.flags & LCS_PCG_ROWS) && !(o.flags & LCS_PCG_PLAIN)) {
        if (P->rows_capacity < 0) P->rows_capacity = (int)lcs_pcg_rows_capacity();
        int rc = LCS_ERR_CAPACITY;
        if ((int64_t)P->n <= P->rows_capacity) {
            if (A && A->row_ptr) {  // the material matrix as SELL-32: coalesced block loads, slice-resident solve
                if ((rc = csr_to_sell(P->msell, P->n, A, s))) return rc;
                // contacts as SELL-32 for the row-resident kernels; the slice-resident one reads the CSR itself
                const bool cb = B && B->row_ptr &&
                                !((o.flags & LCS_PCG_SINGLE_REDUCTION) && !(o.flags & kPcgNoResident) && lcs_pcg_resident(P));
                if (cb && (rc = csr_to_sell(P->csell, P->n, B, s))) return rc;
                rc = rows_solve(P, d4, 1, P->msell.ptr, P->msell.col, P->msell.val, to_bsr(B), b4, x4, o, stats, s,
                                cb ? P->csell.ptr : nullptr, cb ? P->csell.col : nullptr,
                                cb ? P->csell.val : nullptr, cb ? P->csell.ok : nullptr);
            } else {
                rc = rows_solve(P, d4, 0, nullptr, nullptr, nullptr, to_bsr(B), b4, x4, o, stats, s);
            }
        }
        if (rc != LCS_ERR_CAPACITY) return rc;  // too many rows for one thread each: persistent solve below
    }
    if (o.flags & LCS_PCG_PLAIN) {
        if (o.flags & LCS_PCG_FP64_DOTS) return plain_solve<double>(P, d4, to_bsr(A), to_bsr(B), b4, x4, o, stats, s);
        return plain_solve<float>(P, d4, to_bsr(A), to_bsr(B), b4, x4, o, stats, s);
    }
    FusedArgs a;
    a.n = P->n;
    a.diag = d4;
    a.A = to_bsr(A);
    a.B = to_bsr(B);
    a.b = b4;
    a.x = x4;
    a.r = P->r; a.z = P->z; a.p = P->p; a.q = P->q; a.minv = P->minv;
    a.part = P->part;
    a.bar_count = P->bar;
    a.bar_gen = P->bar + 1;
    a.max_iter = o.max_iter;
    a.rel_tol = o.rel_tol;
    a.abs_rz_tol = o.abs_rz_tol;
    a.check_every = o.check_every;
    a.fp64 = (o.flags & LCS_PCG_FP64_DOTS) ? 1 : 0;
    a.stats = P->d_stats;
    LCS_CUDA_TRY(cudaMemsetAsync(P->d_stats, 0, sizeof(lcs_pcg_stats), s));
    LCS_CUDA_TRY(cudaMemsetAsync(P->bar, 0, sizeof(unsigned), s));
    void* args[] = {&a};
    LCS_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_pcg_fused<kRowLanes>, dim3(P->fused_grid), dim3(kFusedThreads), args,
                                             0, s));
    lcs_count_launch();
    if (stats && !(o.flags & LCS_PCG_NO_STATS)) {
        LCS_CUDA_TRY(cudaMemcpyAsync(stats, P->d_stats, sizeof(lcs_pcg_stats), cudaMemcpyDeviceToHost, s));
        LCS_CUDA_TRY(cudaStreamSynchronize(s));
        if (stats->status != LCS_OK) return lcs_fail(stats->status, "lcs_pcg_solve: fused solve failed");
    }
    return LCS_OK;
}

// ------------------------------------------------------------------------------------------
// Allocation-free PCG solve.
//
// Some callers cannot allocate device memory at solve time: cudaMalloc / cudaFree synchronise
// the whole device, which a fixed-latency simulation loop cannot afford, and a host framework
// that hands the whole GPU to its own pool allocator leaves nothing for a library to
// cudaMalloc.  lcs_pcg_solve_noalloc runs the same persistent solve as lcs_pcg_solve, but its
// working vectors live in one file-scope device array, g_pcg_scratch (7.3 MB), so it needs no
// handle and allocates nothing itself.
//
// When the array's memory is taken: the device memory of a module's __device__ variables is
// reserved when that module is loaded on a device.  Under CUDA's default lazy module loading
// (CUDA_MODULE_LOADING=LAZY) that happens on the first use of this file's module on that device:
// the first call of this entry point (its set-up takes the array's address) or the first launch
// of any PCG kernel of the library, whichever comes first.  It is held until the process exits.
// A caller that hands the device's memory to its own pool must therefore make one call (or use
// any PCG entry point) on each device before the pool takes the memory; if the memory is gone
// by then, the set-up reports LCS_ERR_CAPACITY.
//
// Limits and sharing rules:
//  * at most kNoAllocMaxRows (65,536) block rows; larger systems are rejected with
//    LCS_ERR_CAPACITY;
//  * every call on a device shares the one array and leaves the last call's contents in it:
//    two calls whose work overlaps on the GPU (different streams, or different host threads)
//    race on it and give wrong results, so the caller must order them;
//  * the first call on each device resolves the array's device address with
//    cudaGetSymbolAddress (host code cannot use the symbol itself as a pointer) and caches it
//    for the life of the process; make that first call before any stream capture.  The cache
//    does not survive cudaDeviceReset (the address belongs to the old context): do not call
//    this entry point on a device after resetting it.
// ------------------------------------------------------------------------------------------
constexpr uint32_t kNoAllocMaxRows = 65536;
constexpr uint32_t kNoAllocMaxBlocks = 1024;
constexpr size_t kNaVec = 16ull * kNoAllocMaxRows;              // one float4 per row
constexpr size_t kNaOffR = 0, kNaOffZ = kNaVec, kNaOffP = 2 * kNaVec, kNaOffQ = 3 * kNaVec;
constexpr size_t kNaOffMinv = 4 * kNaVec;                        // three float4 per row
constexpr size_t kNaOffPart = 7 * kNaVec;                        // 3 doubles per block
constexpr size_t kNaOffBar = kNaOffPart + 24ull * kNoAllocMaxBlocks;
constexpr size_t kNaOffStats = kNaOffBar + 256;
constexpr size_t kNaBytes = kNaOffStats + 256;

static __device__ __align__(256) unsigned char g_pcg_scratch[kNaBytes];

namespace {
struct NoAllocDevice {
    unsigned char* base = nullptr;
    int grid = 0;
};
std::mutex g_noalloc_mutex;
NoAllocDevice g_noalloc[64];
}  // namespace

extern "C" int lcs_pcg_solve_noalloc(uint32_t n, const float* diag, const lcs_bsr* A, const lcs_bsr* B,
                                     const float* b, float* x, const lcs_pcg_opts* opts, lcs_pcg_stats* stats,
                                     lcs_stream stream)
{
    if (!diag || !b || !x || n == 0) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_noalloc: bad argument");
    if (n > kNoAllocMaxRows)
        return lcs_fail(LCS_ERR_CAPACITY, "lcs_pcg_solve_noalloc: more than 65536 block rows (static scratch limit)");
    if ((A && A->n_rows != n) || (B && B->n_rows != n))
        return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_noalloc: row count mismatch");
    lcs_pcg_opts o = opts ? *opts : lcs_pcg_opts{100, 1e-4f, 1e-10f, 25, 0};  // the defaults of lcs_pcg_solve
    if (o.flags & (LCS_PCG_PLAIN | LCS_PCG_ROWS | LCS_PCG_SINGLE_REDUCTION))
        return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_noalloc: only the fused solve is allocation-free "
                                         "(LCS_PCG_PLAIN, LCS_PCG_ROWS and LCS_PCG_SINGLE_REDUCTION are rejected)");
    if (o.check_every <= 0) o.check_every = 1;
    int dev = 0;
    LCS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_noalloc: device index out of range");
    NoAllocDevice nd;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc[dev].base) {  // one-time set-up on this device, with it current
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();  // do not leave the error for an unrelated later check to find
                static thread_local char msg[256];
                const bool oom = e == cudaErrorMemoryAllocation;
                std::snprintf(msg, sizeof(msg), "lcs_pcg_solve_noalloc: set-up could not reserve the %zu-byte static "
                              "scratch on device %d (cudaGetSymbolAddress: %s)%s", kNaBytes, dev,
                              cudaGetErrorString(e), oom ? "; make the first call before a pool takes the memory" : "");
                return lcs_fail(oom ? LCS_ERR_CAPACITY : LCS_ERR_CUDA, msg);
            }
            int sms = 0, per_sm = 0;
            LCS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            LCS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_fused<kRowLanes>, kFusedThreads, 0));
            int grid = sms * (per_sm > 0 ? 1 : 0);
            if (grid <= 0 || grid > (int)kNoAllocMaxBlocks)
                return lcs_fail(LCS_ERR_CUDA, "lcs_pcg_solve_noalloc: no co-resident launch shape");
            g_noalloc[dev].base = static_cast<unsigned char*>(p);
            g_noalloc[dev].grid = grid;
        }
        nd = g_noalloc[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* base = nd.base;
    FusedArgs a;
    a.n = n;
    a.diag = reinterpret_cast<const float4*>(diag);
    a.A = to_bsr(A);
    a.B = to_bsr(B);
    a.b = reinterpret_cast<const float4*>(b);
    a.x = reinterpret_cast<float4*>(x);
    a.r = reinterpret_cast<float4*>(base + kNaOffR);
    a.z = reinterpret_cast<float4*>(base + kNaOffZ);
    a.p = reinterpret_cast<float4*>(base + kNaOffP);
    a.q = reinterpret_cast<float4*>(base + kNaOffQ);
    a.minv = reinterpret_cast<float4*>(base + kNaOffMinv);
    a.part = reinterpret_cast<double*>(base + kNaOffPart);
    a.bar_count = reinterpret_cast<unsigned*>(base + kNaOffBar);
    a.bar_gen = reinterpret_cast<unsigned*>(base + kNaOffBar) + 1;
    a.max_iter = o.max_iter;
    a.rel_tol = o.rel_tol;
    a.abs_rz_tol = o.abs_rz_tol;
    a.check_every = o.check_every;
    a.fp64 = (o.flags & LCS_PCG_FP64_DOTS) ? 1 : 0;
    a.stats = reinterpret_cast<lcs_pcg_stats*>(base + kNaOffStats);
    // the barrier arrival counter and the stats must start at zero; the rest is written
    // before it is read
    LCS_CUDA_TRY(cudaMemsetAsync(a.bar_count, 0, sizeof(unsigned), s));
    LCS_CUDA_TRY(cudaMemsetAsync(a.stats, 0, sizeof(lcs_pcg_stats), s));
    void* args[] = {&a};
    LCS_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_pcg_fused<kRowLanes>, dim3(nd.grid), dim3(kFusedThreads),
                                             args, 0, s));
    lcs_count_launch();
    if (stats && !(o.flags & LCS_PCG_NO_STATS)) {
        LCS_CUDA_TRY(cudaMemcpyAsync(stats, a.stats, sizeof(lcs_pcg_stats), cudaMemcpyDeviceToHost, s));
        LCS_CUDA_TRY(cudaStreamSynchronize(s));
        if (stats->status != LCS_OK) return lcs_fail(stats->status, "lcs_pcg_solve_noalloc: solve failed");
    }
    return LCS_OK;
}

template <class Launch>
static int solve_batch_auto(lcs_pcg* P, uint32_t n_scenes, const uint32_t* host_row_offsets, Launch& launch,
                            cudaStream_t s0);

extern "C" int lcs_pcg_batch_tuning(const lcs_pcg* p, uint32_t* chunks_per_cta, float* solve_ms)
{
    if (!p) return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_batch_tuning: null handle");
    if (chunks_per_cta) *chunks_per_cta = p->tuned_target;
    if (solve_ms) *solve_ms = p->tuned_ms;
    return LCS_OK;
}

extern "C" int lcs_pcg_solve_batch(lcs_pcg* P, uint32_t n_scenes, const uint32_t* row_offsets, const uint32_t* host_row_offsets,
                                   const uint32_t* active, const float* diag, const lcs_bsr* A, const lcs_bsr* B,
                                   const float* b, float* x, const lcs_pcg_opts* opts, lcs_pcg_stats* stats_per_scene,
                                   int cluster, lcs_stream stream)
{
    if (!P || !row_offsets || !host_row_offsets || !diag || !b || !x || !stats_per_scene || n_scenes == 0)
        return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_batch: bad argument");
    const uint32_t* host_row_end = host_row_offsets + n_scenes;
    if (*host_row_end > P->n || (A && A->n_rows != P->n) || (B && B->n_rows != P->n))
        return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_batch: row count mismatch");
    if (cluster != 0 && cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8 && cluster != 16)
        return lcs_fail(LCS_ERR_INVALID, "lcs_pcg_solve_batch: cluster size must be 0 (auto), 1, 2, 4, 8 or 16");
    lcs_pcg_opts o = opts ? *opts : lcs_pcg_opts{100, 1e-4f, 1e-10f, 1, 0};
    if (o.check_every <= 0) o.check_every = 1;
    const size_t chunks = (size_t)(*host_row_end >> 8) + n_scenes + 1;
    if (chunks > P->cpart_cap) {
        if (P->cpart) cudaFree(P->cpart);
        P->cpart = nullptr;
        P->cpart_cap = 0;
        LCS_CUDA_TRY(cudaMalloc((void**)&P->cpart, 4 * sizeof(double) * chunks));
        P->cpart_cap = chunks;
    }
    BatchArgs a;
    a.roff = row_offsets;
    a.active = active;
    a.diag = reinterpret_cast<const float4*>(diag);
    a.A = to_bsr(A);
    a.B = to_bsr(B);
    a.b = reinterpret_cast<const float4*>(b);
    a.x = reinterpret_cast<float4*>(x);
    a.r = P->r; a.z = P->z; a.p = P->p; a.q = P->q; a.minv = P->minv;
    a.cpart = P->cpart;
    a.max_iter = o.max_iter;
    a.rel_tol = o.rel_tol;
    a.abs_rz_tol = o.abs_rz_tol;
    a.check_every = o.check_every;
    a.fp64 = (o.flags & LCS_PCG_FP64_DOTS) ? 1 : 0;
    a.stats = stats_per_scene;
    a.scenes = nullptr;
    auto launch = [&](int C, uint32_t clusters, const uint32_t* scene_list, cudaStream_t st) -> cudaError_t {
        if (C == 16) {
            const cudaError_t e = cudaFuncSetAttribute(k_pcg_batch, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
        }
        BatchArgs b = a;
        b.scenes = scene_list;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(clusters * (uint32_t)C);
        cfg.blockDim = dim3(kBatchThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, k_pcg_batch, b);
    };
    cudaStream_t s0 = (cudaStream_t)stream;
    if (cluster != 0) {
        LCS_CUDA_TRY(launch(cluster, n_scenes, nullptr, s0));
        lcs_count_launch();
        return LCS_OK;
    }
    // auto: every scene gets the smallest cluster (1..16 CTAs) that leaves it at most `target` chunks of 256
    // rows per CTA; one launch per cluster size, on forked streams so that the classes run side by side.
    // The target is tuned on the first solve of the handle: the same system is solved with each candidate
    // (2, 4, 8, 16 chunks per CTA; a scene's solution does not depend on its cluster size) and the fastest
    // is kept.
    if (P->tuned_target == 0) {
        P->tuned_target = 8;  // the untimed default while tuning (and if a timing fails)
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
            float best = 0.0f;
            uint32_t best_target = 8;
            for (uint32_t target : {2u, 4u, 8u, 16u}) {
                P->tuned_target = target;
                LCS_CUDA_TRY(cudaEventRecord(e0, s0));
                const int rc = solve_batch_auto(P, n_scenes, host_row_offsets, launch, s0);
                if (rc != LCS_OK) return rc;
                LCS_CUDA_TRY(cudaEventRecord(e1, s0));
                LCS_CUDA_TRY(cudaEventSynchronize(e1));
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (best == 0.0f || ms < best) {
                    best = ms;
                    best_target = target;
                }
            }
            P->tuned_target = best_target;
            P->tuned_ms = best;
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    return solve_batch_auto(P, n_scenes, host_row_offsets, launch, s0);
}

template <class Launch>
static int solve_batch_auto(lcs_pcg* P, uint32_t n_scenes, const uint32_t* host_row_offsets, Launch& launch,
                            cudaStream_t s0)
{
    std::vector<uint32_t> lists[5];
    for (uint32_t sc = 0; sc < n_scenes; ++sc) {
        const uint32_t chunks = (host_row_offsets[sc + 1] - host_row_offsets[sc] + 255) / 256;
        int k = 0;
        while (k < 4 && chunks > P->tuned_target << k) ++k;
        lists[k].push_back(sc);
    }
    std::vector<uint32_t> flat;
    size_t start[6] = {0};
    for (int k = 0; k < 5; ++k) {
        start[k] = flat.size();
        flat.insert(flat.end(), lists[k].begin(), lists[k].end());
    }
    start[5] = flat.size();
    if (flat.size() > P->class_cap) {
        if (P->class_scenes) cudaFree(P->class_scenes);
        P->class_scenes = nullptr;
        P->class_cap = 0;
        LCS_CUDA_TRY(cudaMalloc((void**)&P->class_scenes, 4 * flat.size()));
        P->class_cap = flat.size();
        P->class_host.clear();
    }
    if (P->class_host != flat) {  // scene lists change only with the scenes' sizes
        LCS_CUDA_TRY(cudaMemcpyAsync(P->class_scenes, flat.data(), 4 * flat.size(), cudaMemcpyHostToDevice, s0));
        LCS_CUDA_TRY(cudaStreamSynchronize(s0));
        P->class_host = flat;
    }
    if (!P->class_fork) {
        LCS_CUDA_TRY(cudaEventCreateWithFlags(&P->class_fork, cudaEventDisableTiming));
        for (int k = 0; k < 5; ++k) {
            LCS_CUDA_TRY(cudaStreamCreateWithFlags(&P->class_stream[k], cudaStreamNonBlocking));
            LCS_CUDA_TRY(cudaEventCreateWithFlags(&P->class_join[k], cudaEventDisableTiming));
        }
    }
    LCS_CUDA_TRY(cudaEventRecord(P->class_fork, s0));
    for (int k = 0; k < 5; ++k) {
        const uint32_t m = (uint32_t)(start[k + 1] - start[k]);
        if (m == 0) continue;
        LCS_CUDA_TRY(cudaStreamWaitEvent(P->class_stream[k], P->class_fork, 0));
        LCS_CUDA_TRY(launch(1 << k, m, P->class_scenes + start[k], P->class_stream[k]));
        lcs_count_launch();
        LCS_CUDA_TRY(cudaEventRecord(P->class_join[k], P->class_stream[k]));
        LCS_CUDA_TRY(cudaStreamWaitEvent(s0, P->class_join[k], 0));
    }
    return LCS_OK;
}
