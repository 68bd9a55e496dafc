// material.cu -- per-element cloth energies behind the C ABI: the reference's evaluate kernels
// with their per-element output layout (fn_evaluate_spring / fn_evaluate_stretch_face /
// fn_evaluate_bending, Solver/SimulationSolver/newton_solver.cpp:1002-1175) and the elastic
// energy of the line search (fn_calc_energy_*, Solver/SimulationSolver/solver_interface.cpp:505-728)
// summed in FP64.  The Newton loop does not go through these: it evaluates the same device
// functions (material.cuh) and adds the results straight into b, the diagonal and the material
// BSR (csrc/newton.cu), without the per-element arrays and the gather pass of the reference's
// assembly kernels (newton_solver.cpp:705-814).
#include <cuda_runtime.h>

#include "lcs_internal.h"
#include "material.cuh"

using namespace lcs;

namespace {

__device__ __forceinline__ void st3(float4* p, v3 a) { *p = make_float4(a.x, a.y, a.z, 0.0f); }
// 3x3 block (column-major [3 c + r]) to a float3x3 record (three 16-byte columns); transposed if t
__device__ __forceinline__ void st33(float4* p, const float* K, bool t)
{
#pragma unroll
    for (int c = 0; c < 3; ++c)
        p[c] = t ? make_float4(K[c], K[3 + c], K[6 + c], 0.0f) : make_float4(K[3 * c], K[3 * c + 1], K[3 * c + 2], 0.0f);
}

__global__ void k_eval_springs(uint32_t n, const float4* __restrict__ x, const uint2* __restrict__ edges,
                               const float* __restrict__ rest_len, const float* __restrict__ stiff, float4* grad,
                               float4* hess)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint2 ed = edges[e];
        const v3 p0 = ld3(x, ed.x), p1 = ld3(x, ed.y);
        const v3 d = p0 - p1;
        const float l = fmx(sqrtf(dot3(d, d)), 1.19209290E-7f);
        const float k = stiff[e], L = rest_len[e];
        const float C = l - L, il = 1.0f / l, il2 = il * il;
        const v3 g = mk3(k * d.x * il * C, k * d.y * il * C, k * d.z * il * C);
        st3(&grad[2 * (size_t)e], g);
        st3(&grad[2 * (size_t)e + 1], neg3(g));
        const float a = k * il2, c = k * fmx(1.0f - L * il, 0.0f);
        const float dd[3] = {d.x, d.y, d.z};
        float H[9], N[9];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                H[3 * cc + r] = a * dd[r] * dd[cc] + c * ((r == cc ? 1.0f : 0.0f) - il2 * dd[r] * dd[cc]);
                N[3 * cc + r] = -H[3 * cc + r];
            }
        float4* o = hess + 12 * (size_t)e;  // 4 blocks: (0,0) (1,1) (0,1) (1,0)
        st33(o, H, false);
        st33(o + 3, H, false);
        st33(o + 6, N, false);
        st33(o + 9, N, false);
    }
}

__global__ void k_eval_stretch_faces(uint32_t n, const float4* __restrict__ x, const uint4* __restrict__ faces,
                                     const float4* __restrict__ dm, const float* __restrict__ area,
                                     const float2* __restrict__ mu_lambda, float4* grad, float4* hess)
{
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
        const uint4 fc = faces[f];
        const float2 ml = mu_lambda[f];
        Bw98Out o;
        bw98_face(ld3(x, fc.x), ld3(x, fc.y), ld3(x, fc.z), dm[f], ml.x, ml.y, area[f], o);
#pragma unroll
        for (int a = 0; a < 3; ++a) st3(&grad[3 * (size_t)f + a], o.g[a]);
        // blocks: (0,0) (1,1) (2,2), then (0,1) (0,2) (1,0) (1,2) (2,0) (2,1) (row vertex, column vertex)
        float4* h = hess + 27 * (size_t)f;
        st33(h + 0, o.K[0], false);
        st33(h + 3, o.K[1], false);
        st33(h + 6, o.K[2], false);
        st33(h + 9, o.K[3], false);
        st33(h + 12, o.K[4], false);
        st33(h + 15, o.K[3], true);
        st33(h + 18, o.K[5], false);
        st33(h + 21, o.K[4], true);
        st33(h + 24, o.K[5], true);
    }
}

__global__ void k_eval_bending(uint32_t n, const float4* __restrict__ x, const uint4* __restrict__ st,
                               const float* __restrict__ rest_angle, const float* __restrict__ hbar,
                               const float* __restrict__ stiffness, float scaling, float4* grad, float4* hess)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint4 e = st[s];
        v3 g[4];
        const float theta = dihedral_angle_grad(ld3(x, e.x), ld3(x, e.y), ld3(x, e.z), ld3(x, e.w), g);
        const float stiff = stiffness[s] * scaling * hbar[s];
        const float sd = stiff * (theta - rest_angle[s]);
#pragma unroll
        for (int i = 0; i < 4; ++i) st3(&grad[4 * (size_t)s + i], sd * g[i]);
        // blocks stiff g_i g_j^T: (i, i) for i = 0..3, then (i, j), i != j, row-major
        float4* h = hess + 48 * (size_t)s;
        int k = 4;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float gi[3] = {g[i].x, g[i].y, g[i].z}, gj[3] = {g[j].x, g[j].y, g[j].z};
                float K[9];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < 3; ++r) K[3 * c + r] = stiff * (gi[r] * gj[c]);
                st33(h + 3 * (i == j ? i : k), K, false);
                if (i != j) ++k;
            }
    }
}

__device__ __forceinline__ void warp_add_f64(double* dst, double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane_id() == 0 && v != 0.0) atomicAdd(dst, v);
}

// energy terms: [0] inertia (fn_calc_energy_inertia), [1] springs, [2] stretch faces, [3] bending
__global__ void k_material_energy(lcs_cloth_elements m, const float4* __restrict__ x, const float4* __restrict__ xt,
                                  float dt, float dirichlet, double* out)
{
    const uint32_t n = max(max(m.n_verts, m.n_springs), max(m.n_stretch_faces, m.n_bending));
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n_round = (n + stride - 1) / stride * stride;  // all lanes take the same trips
    double e[4] = {0.0, 0.0, 0.0, 0.0};
    const float h2inv = 1.0f / (dt * dt);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += stride) {
        if (i < m.n_verts) {
            const v3 d = ld3(x, i) - ld3(xt, i);
            float en = h2inv * dot3(d, d) * m.mass[i] / 2.0f;
            if (m.is_fixed && m.is_fixed[i]) en = dirichlet * en;
            e[0] += (double)en;
        }
        if (i < m.n_springs) {
            const uint2 ed = reinterpret_cast<const uint2*>(m.springs)[i];
            const v3 d = ld3(x, ed.y) - ld3(x, ed.x);
            const float C = sqrtf(dot3(d, d)) - m.spring_rest_len[i];
            e[1] += (double)(0.5f * m.spring_stiffness[i] * C * C);
        }
        if (i < m.n_stretch_faces) {
            const uint4 fc = reinterpret_cast<const uint4*>(m.stretch_faces)[i];
            const float4 dm = reinterpret_cast<const float4*>(m.stretch_dm_inv)[i];
            const float2 ml = reinterpret_cast<const float2*>(m.stretch_mu_lambda)[i];
            const v3 x0 = ld3(x, fc.x), e1 = ld3(x, fc.y) - x0, e2 = ld3(x, fc.z) - x0;
            const v3 Fu = mk3(__fmaf_rn(e2.x, dm.y, e1.x * dm.x), __fmaf_rn(e2.y, dm.y, e1.y * dm.x),
                              __fmaf_rn(e2.z, dm.y, e1.z * dm.x));
            const v3 Fv = mk3(__fmaf_rn(e2.x, dm.w, e1.x * dm.z), __fmaf_rn(e2.y, dm.w, e1.y * dm.z),
                              __fmaf_rn(e2.z, dm.w, e1.z * dm.z));
            const float su = sqrtf(dot3(Fu, Fu)) - 1.0f, sv = sqrtf(dot3(Fv, Fv)) - 1.0f, i6 = dot3(Fu, Fv);
            const float en = 0.5f * ml.x * (su * su + sv * sv) + 0.5f * ml.y * (i6 * i6);
            e[2] += (double)(m.stretch_area[i] * en);
        }
        if (i < m.n_bending) {
            const uint4 st = reinterpret_cast<const uint4*>(m.bending_edges)[i];
            v3 g[4];
            const float theta = dihedral_angle_grad(ld3(x, st.x), ld3(x, st.y), ld3(x, st.z), ld3(x, st.w), g);
            const float d = theta - m.bending_rest_angle[i];
            e[3] += (double)(0.5f * m.bending_stiffness[i] * m.bending_scaling * m.bending_hbar[i] * d * d);
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) warp_add_f64(out + k, e[k]);
}

int launch_check(const char* what)
{
    lcs_count_launch();
    return cudaGetLastError() == cudaSuccess ? LCS_OK : lcs_fail(LCS_ERR_CUDA, what);
}

}  // namespace

extern "C" int lcs_eval_springs(const float* x, const uint32_t* edges, const float* rest_len, const float* stiffness,
                                uint32_t n, float* gradients, float* hessians, lcs_stream stream)
{
    if (n == 0) return LCS_OK;
    if (!x || !edges || !rest_len || !stiffness || !gradients || !hessians)
        return lcs_fail(LCS_ERR_INVALID, "lcs_eval_springs: null argument");
    k_eval_springs<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        n, reinterpret_cast<const float4*>(x), reinterpret_cast<const uint2*>(edges), rest_len, stiffness,
        reinterpret_cast<float4*>(gradients), reinterpret_cast<float4*>(hessians));
    return launch_check("lcs_eval_springs: launch failed");
}

extern "C" int lcs_eval_stretch_faces(const float* x, const uint32_t* faces, const float* dm_inv, const float* rest_area,
                                      const float* mu_lambda, uint32_t n, float* gradients, float* hessians,
                                      lcs_stream stream)
{
    if (n == 0) return LCS_OK;
    if (!x || !faces || !dm_inv || !rest_area || !mu_lambda || !gradients || !hessians)
        return lcs_fail(LCS_ERR_INVALID, "lcs_eval_stretch_faces: null argument");
    k_eval_stretch_faces<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
        n, reinterpret_cast<const float4*>(x), reinterpret_cast<const uint4*>(faces),
        reinterpret_cast<const float4*>(dm_inv), rest_area, reinterpret_cast<const float2*>(mu_lambda),
        reinterpret_cast<float4*>(gradients), reinterpret_cast<float4*>(hessians));
    return launch_check("lcs_eval_stretch_faces: launch failed");
}

extern "C" int lcs_eval_bending(const float* x, const uint32_t* stencils, const float* rest_angle, const float* rest_hbar,
                                const float* stiffness, float scaling, uint32_t n, float* gradients, float* hessians,
                                lcs_stream stream)
{
    if (n == 0) return LCS_OK;
    if (!x || !stencils || !rest_angle || !rest_hbar || !stiffness || !gradients || !hessians)
        return lcs_fail(LCS_ERR_INVALID, "lcs_eval_bending: null argument");
    k_eval_bending<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
        n, reinterpret_cast<const float4*>(x), reinterpret_cast<const uint4*>(stencils), rest_angle, rest_hbar,
        stiffness, scaling, reinterpret_cast<float4*>(gradients), reinterpret_cast<float4*>(hessians));
    return launch_check("lcs_eval_bending: launch failed");
}

extern "C" int lcs_material_energy(const lcs_cloth_elements* m, const float* x, const float* x_tilde, float dt,
                                   float stiffness_dirichlet, double* energy, lcs_stream stream)
{
    if (!m || !x || !energy || (m->n_verts && (!x_tilde || !m->mass)) ||
        (m->n_springs && (!m->springs || !m->spring_rest_len || !m->spring_stiffness)) ||
        (m->n_stretch_faces && (!m->stretch_faces || !m->stretch_dm_inv || !m->stretch_area || !m->stretch_mu_lambda)) ||
        (m->n_bending && (!m->bending_edges || !m->bending_rest_angle || !m->bending_hbar || !m->bending_stiffness)))
        return lcs_fail(LCS_ERR_INVALID, "lcs_material_energy: incomplete element description");
    cudaStream_t s = (cudaStream_t)stream;
    LCS_CUDA_TRY(cudaMemsetAsync(energy, 0, 4 * sizeof(double), s));
    const uint32_t n = std::max(std::max(m->n_verts, m->n_springs), std::max(m->n_stretch_faces, m->n_bending));
    if (n == 0) return LCS_OK;
    k_material_energy<<<grid_for(n, 256), 256, 0, s>>>(*m, reinterpret_cast<const float4*>(x),
                                                      reinterpret_cast<const float4*>(x_tilde), dt,
                                                      stiffness_dirichlet, energy);
    return launch_check("lcs_material_energy: launch failed");
}
