// newton.cu -- the Newton loop around the contact path (NewtonSolver::physics_step_GPU,
// Solver/SimulationSolver/newton_solver.cpp:4051-4345) and the glue the reference keeps in
// NewtonSolver: broad/narrow phase drivers with resize-and-retry, CCD line search, apply dx
// (newton_solver.cpp:3174-3375, 3685-3884), plus the per-vertex producers that feed it
// (inertia with Dirichlet pinning, edge springs, quadratic bending; newton_solver.cpp:819-851,
// 1003-1175; init_sim_data.cpp:455-480).
//
// Two executions of the same algorithm:
//  * fused (default): device Morton sort, leaf update fused with the refit, candidate and pair
//    counts kept on the device, the whole PCG solve in one persistent launch, and a single
//    host synchronisation per Newton iteration (a 64-byte status read from pinned memory);
//    a capacity overflow anywhere in the iteration is detected there and the iteration is
//    re-run with grown buffers;
//  * plain (LCS_NEWTON_PLAIN): the reference's dispatch structure -- host Morton sort,
//    separate leaf-update and refit launches, one kernel per PCG operation with a host check
//    of r.z every check_every iterations, and the reference's host read-backs (broad counts,
//    narrow counts, adjacency prescan, triplet sort, TOI, positions) -- used as the
//    one-scene-at-a-time GPU comparator.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <utility>
#include <chrono>
#include <thread>
#include <vector>

#include "lcs_common.cuh"
#include "lcs_internal.h"
#include "lcs_geom.cuh"
#include "material.cuh"
#include "abd.cuh"
#include "radix_sort.cuh"

using namespace lcs;

namespace {

struct Status {
    uint32_t cnt[6];  // 0 DCD vf, 1 DCD ee, 2 contact pairs, 3 CCD vf, 4 CCD ee, 5 a CCD traversal ended early
    float toi;
    float max_dx;     // max_v |dx_v| (before the step bound)
    float dirichlet;  // max over pinned vertices |x - x_tilde| after the step
    int32_t pcg_iters;
    float pcg_rel;
    int32_t pcg_status;
    float alpha;      // step length applied: the CCD bound, or the energy line search's choice
    int32_t ls_iters; // halvings of the accepted step length (energy line search)
    int32_t ls_state; // energy line search: 0 not run, 1 decided, 2 undecided after this round, 3 failed
    float pad;
};

// animation of a group of pinned vertices (FixedPointAnimationInfo::fn_affine_position,
// Solver/Initializer/init_mesh_data.h:61-92): mode bit 1 scale by (s t), bit 0 rotate about the axis
// through the centre by omega t, bit 2 translate by (tr t), in that order
struct Anim {
    float cx, cy, cz, ax, ay, az, omega, mode;
    float tx, ty, tz, sx, sy, sz, pad0, pad1;
};

// affine bodies on the device (body == nullptr: none).  slot[v] = j for the j-th DOF slot of a body
// (holding p, a0, a1, a2), -1 otherwise; a vertex with a body id and slot -1 is a rigid mesh vertex.
struct AbdDev {
    const uint32_t* body;
    const int8_t* slot;
    const float4* model_x;
    const uint32_t* body_dof;
    const uint8_t* fixed;  // per body
};

__device__ __forceinline__ bool is_rigid(const AbdDev& a, uint32_t i)
{
    return a.body && a.body[i] != kInvalid && a.slot[i] < 0;
}

// x0 + alpha dx for vertex i; a rigid vertex follows its body: p + A x_bar with q = q0 + alpha dq
__device__ __forceinline__ float4 stepped(const AbdDev& a, uint32_t i, const float4* __restrict__ x0,
                                          const float4* __restrict__ dx, float alpha)
{
    if (is_rigid(a, i)) {
        const uint32_t d = a.body_dof[a.body[i]];
        v3 q[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float4 p = x0[d + j], e = dx[d + j];
            q[j] = mk3(p.x + alpha * e.x, p.y + alpha * e.y, p.z + alpha * e.z);
        }
        const v3 r = affine_apply(q[0], q[1], q[2], q[3], a.model_x[i]);
        return make_float4(r.x, r.y, r.z, 0.0f);
    }
    const float4 p = x0[i], e = dx[i];
    return make_float4(p.x + alpha * e.x, p.y + alpha * e.y, p.z + alpha * e.z, 0.0f);
}

__device__ __forceinline__ void atomic_max_pos(float* a, float v) { atomicMax(reinterpret_cast<int*>(a), __float_as_int(v)); }

__global__ void k_reset_status(Status* s)
{
    if (threadIdx.x < 6) s->cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        s->toi = 1.0f;
        s->max_dx = 0.0f;
        s->dirichlet = 0.0f;
    }
}

// targets of animated pinned vertices at time t (WorldData::get_fixed_point_target_positions,
// init_mesh_data.cpp:272-297)
__global__ void k_targets(uint32_t n, const float4* __restrict__ rest, const int8_t* __restrict__ group,
                          const Anim* __restrict__ anim, float t, float4* __restrict__ target)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p = rest[i];
        const int g = group ? group[i] : -1;
        const int mode = g >= 0 ? (int)anim[g].mode : 0;
        if (g >= 0 && (mode & 2)) {
            const Anim A = anim[g];
            p.x = (A.sx * t) * p.x;
            p.y = (A.sy * t) * p.y;
            p.z = (A.sz * t) * p.z;
        }
        if (g >= 0 && (mode & 1)) {
            const Anim A = anim[g];
            const float ang = A.omega * t;
            const float c = cosf(ang), s = sinf(ang);
            const float px = p.x - A.cx, py = p.y - A.cy, pz = p.z - A.cz;
            const float d = A.ax * px + A.ay * py + A.az * pz;
            const float kx = A.ay * pz - A.az * py, ky = A.az * px - A.ax * pz, kz = A.ax * py - A.ay * px;
            p.x = A.cx + px * c + kx * s + A.ax * d * (1.0f - c);
            p.y = A.cy + py * c + ky * s + A.ay * d * (1.0f - c);
            p.z = A.cz + pz * c + kz * s + A.az * d * (1.0f - c);
        }
        if (g >= 0 && (mode & 4)) {
            const Anim A = anim[g];
            p.x = p.x + A.tx * t;
            p.y = p.y + A.ty * t;
            p.z = p.z + A.tz * t;
        }
        target[i] = p;
    }
}

// physics_step_prev_operation + fn_predict_position (solver_interface.cpp:130-162,
// newton_solver.cpp:576-604): pinned vertices get v = (target - x) / dt
__global__ void k_predict(uint32_t n, float dt, float gx, float gy, float gz, const uint8_t* __restrict__ pinned,
                          const float4* __restrict__ target, const float4* __restrict__ x, float4* __restrict__ v,
                          float4* __restrict__ x_step_start, float4* __restrict__ x_tilde, AbdDev abd)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 xp = x[i];
        float4 vp = v[i];
        float3 vpred;
        const int slot = abd.body ? abd.slot[i] : -1;
        if (slot >= 0) {
            // fn_abd_predict_position (newton_solver.cpp:640-676): gravity on the translation only, none
            // for a fixed body
            const bool acc = slot == 0 && !abd.fixed[abd.body[i]];
            vpred = acc ? make_float3(vp.x + dt * gx, vp.y + dt * gy, vp.z + dt * gz) : make_float3(vp.x, vp.y, vp.z);
        } else if (is_rigid(abd, i)) {
            vpred = make_float3(0.0f, 0.0f, 0.0f);  // x_tilde of rigid vertices: k_abd_rigid_tilde
        } else if (pinned && pinned[i]) {
            const float4 tg = target[i];
            vp = make_float4((tg.x - xp.x) / dt, (tg.y - xp.y) / dt, (tg.z - xp.z) / dt, 0.0f);
            v[i] = vp;
            vpred = make_float3(vp.x, vp.y, vp.z);
        } else {
            vpred = make_float3(vp.x + dt * gx, vp.y + dt * gy, vp.z + dt * gz);
        }
        x_step_start[i] = xp;
        x_tilde[i] = make_float4(xp.x + dt * vpred.x, xp.y + dt * vpred.y, xp.z + dt * vpred.z, 0.0f);
    }
}

// fn_evaluate_inertia (+ fn_evaluate_ground_collision when the floor is on), newton_solver.cpp:819-951;
// also x_iter_start = x and dx = 0
__global__ void k_inertia(uint32_t n, float h, float dirichlet, const float* __restrict__ mass,
                          const uint8_t* __restrict__ pinned, const float4* __restrict__ x,
                          const float4* __restrict__ x_tilde, float4* __restrict__ x_iter_start, float4* __restrict__ b,
                          float4* __restrict__ diag, int use_floor, float floor_y, float kappa,
                          const float* __restrict__ vert_area, const float* __restrict__ dhat,
                          const float* __restrict__ offset, AbdDev abd)
{
    const float h2inv = 1.0f / (h * h);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (abd.body && abd.body[i] != kInvalid) {
            // a rigid mesh vertex's row is inert (identity, zero right-hand side); a DOF slot's row is
            // written by k_abd_body
            const float one = abd.slot[i] < 0 ? 1.0f : 0.0f;
            x_iter_start[i] = x[i];
            b[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            diag[3 * i + 0] = make_float4(one, 0.0f, 0.0f, 0.0f);
            diag[3 * i + 1] = make_float4(0.0f, one, 0.0f, 0.0f);
            diag[3 * i + 2] = make_float4(0.0f, 0.0f, one, 0.0f);
            continue;
        }
        const float4 xk = x[i], xt = x_tilde[i];
        const float m = mass[i];
        const float s = -m * h2inv;
        float3 g = make_float3(s * (xk.x - xt.x), s * (xk.y - xt.y), s * (xk.z - xt.z));
        float hd = m * h2inv;
        const bool fixed = pinned && pinned[i];
        if (fixed) {
            g = make_float3(g.x + dirichlet * g.x, g.y + dirichlet * g.y, g.z + dirichlet * g.z);
            hd = hd + dirichlet * hd;
        }
        float hyy = hd;
        if (use_floor && !fixed) {
            const float dh = dhat[i], th = offset[i], dist = xk.y - floor_y;
            if (dist - th < dh) {
                const float stiff = kappa * vert_area[i];
                const float d = dist - th;
                const float k1 = stiff * ((dh - d) * (2.0f * logf(d / dh) - dh / d + 1.0f));
                const float q = dh / d;
                const float k2 = stiff * ((q + 2.0f) * q - 2.0f * logf(d / dh) - 3.0f);
                g.y -= k1;
                hyy += k2;
            }
        }
        x_iter_start[i] = xk;
        b[i] = make_float4(g.x, g.y, g.z, 0.0f);
        diag[3 * i + 0] = make_float4(hd, 0.0f, 0.0f, 0.0f);
        diag[3 * i + 1] = make_float4(0.0f, hyy, 0.0f, 0.0f);
        diag[3 * i + 2] = make_float4(0.0f, 0.0f, hd, 0.0f);
    }
}

__device__ __forceinline__ void atomic_add3(float4* p, float x, float y, float z)
{
    float* f = reinterpret_cast<float*>(p);
    atomicAdd(f + 0, x);
    atomicAdd(f + 1, y);
    atomicAdd(f + 2, z);
}

// fn_evaluate_spring + its assembly (newton_solver.cpp:1003-1045): projected spring Hessian
__global__ void k_springs(uint32_t ne, const uint2* __restrict__ edges, const float* __restrict__ rest_len,
                          const float* __restrict__ kper, float k_scalar, const float4* __restrict__ x, float4* b,
                          float4* diag, const uint32_t* __restrict__ slots, uint32_t cs, float* mat_val)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const float k = kper ? kper[e] : k_scalar;
        const uint2 ed = edges[e];
        const float4 p0 = x[ed.x], p1 = x[ed.y];
        const float dx = p0.x - p1.x, dy = p0.y - p1.y, dz = p0.z - p1.z;
        const float l = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1.19209290E-7f);
        const float L = rest_len[e];
        const float C = l - L;
        const float il = 1.0f / l, il2 = il * il;
        const float gx = k * dx * il * C, gy = k * dy * il * C, gz = k * dz * il * C;
        atomic_add3(&b[ed.x], -gx, -gy, -gz);
        atomic_add3(&b[ed.y], gx, gy, gz);
        const float a = k * il2, c = k * fmaxf(1.0f - L * il, 0.0f);
        const float d[3] = {dx, dy, dz};
        float H[9];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int r = 0; r < 3; ++r) H[3 * cc + r] = a * d[r] * d[cc] + c * ((r == cc ? 1.0f : 0.0f) - il2 * d[r] * d[cc]);
        float* D0 = reinterpret_cast<float*>(diag + 3 * (size_t)ed.x);
        float* D1 = reinterpret_cast<float*>(diag + 3 * (size_t)ed.y);
        float* O0 = mat_val + slots[2 * e];  // block bases; component c at c * cs
        float* O1 = mat_val + slots[2 * e + 1];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                atomicAdd(D0 + 4 * cc + r, H[3 * cc + r]);
                atomicAdd(D1 + 4 * cc + r, H[3 * cc + r]);
                atomicAdd(O0 + cs * (3 * cc + r), -H[3 * cc + r]);
                atomicAdd(O1 + cs * (3 * cc + r), -H[3 * cc + r]);
            }
    }
}

// quadratic bending (init_sim_data.cpp:455-480 Q; newton_solver.cpp:3014-3040) measured from the
// rest shape: grad_i = k sum_j Q_ij (x_j - X_j), Hessian block (i, j) = k Q_ij I
__global__ void k_bending(uint32_t nb, const uint4* __restrict__ stencil, const float* __restrict__ Q, float k,
                          const float4* __restrict__ x, const float4* __restrict__ rest, float4* b, float4* diag,
                          const uint32_t* __restrict__ slots, uint32_t cs, float* mat_val)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nb; s += gridDim.x * blockDim.x) {
        const uint4 st = stencil[s];
        const uint32_t v[4] = {st.x, st.y, st.z, st.w};
        float3 u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float4 p = x[v[j]], r = rest[v[j]];
            u[j] = make_float3(p.x - r.x, p.y - r.y, p.z - r.z);
        }
        const float* q = Q + 16 * (size_t)s;
        int t = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float3 g = make_float3(0.f, 0.f, 0.f);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float qij = k * q[4 * i + j];
                g.x += qij * u[j].x;
                g.y += qij * u[j].y;
                g.z += qij * u[j].z;
                if (i == j) {
                    float* D = reinterpret_cast<float*>(diag + 3 * (size_t)v[i]);
                    atomicAdd(D + 0, qij);
                    atomicAdd(D + 5, qij);
                    atomicAdd(D + 10, qij);
                } else {
                    float* O = mat_val + slots[12 * s + t];
                    atomicAdd(O, qij);
                    atomicAdd(O + 4 * cs, qij);
                    atomicAdd(O + 8 * cs, qij);
                    ++t;
                }
            }
            atomic_add3(&b[v[i]], -g.x, -g.y, -g.z);
        }
    }
}

// ---- affine bodies
// x_tilde of rigid mesh vertices from their body's predicted q (used by the Dirichlet check)
__global__ void k_abd_rigid_tilde(uint32_t n, AbdDev abd, float4* __restrict__ x_tilde)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!is_rigid(abd, i)) continue;
        const uint32_t d = abd.body_dof[abd.body[i]];
        const v3 r = affine_apply(ld3(x_tilde, d), ld3(x_tilde, d + 1), ld3(x_tilde, d + 2), ld3(x_tilde, d + 3),
                                  abd.model_x[i]);
        x_tilde[i] = make_float4(r.x, r.y, r.z, 0.0f);
    }
}

// fn_evaluate_abd_inertia + fn_evaluate_abd_orthogonality + fn_material_energy_assembly_affine_body
// (newton_solver.cpp:1176-1330, 705-814): per body, b = -grad and the 4 x 4 blocks of
//   inertia       alpha h^-2 M (x) I, grad_i = alpha h^-2 sum_j M_ij (q_j - q~_j), alpha = 1 (+ dirichlet if fixed)
//   orthogonality kappa V sum_ij (a_i.a_j - delta_ij)^2 on A = [a0 a1 a2] (the reference's gradient and
//                 Hessian blocks: 4 s (sum_j (a_i.a_j) a_j - a_i); 4 s (a_i a_i^T + (a_i.a_i - 1) I +
//                 sum_k a_k a_k^T) on the diagonal, 4 s (a_j a_i^T + (a_i.a_j) I) at (i, j), i < j)
// written into the body's DOF slot rows; off-diagonal blocks (i, j), i != j, row-major in `slots`.
__global__ void k_abd_body(uint32_t nb, const uint32_t* __restrict__ body_dof, const float* __restrict__ mass16,
                           const float* __restrict__ volume, const float* __restrict__ kappa,
                           const uint8_t* __restrict__ fixed, float h2inv, float dirichlet,
                           const float4* __restrict__ x, const float4* __restrict__ x_tilde, float4* b, float4* diag,
                           const uint32_t* __restrict__ slots, uint32_t cs, float* mat_val)
{
    for (uint32_t bi = blockIdx.x * blockDim.x + threadIdx.x; bi < nb; bi += gridDim.x * blockDim.x) {
        const uint32_t d = body_dof[bi];
        v3 q[4], dq[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            q[j] = ld3(x, d + j);
            dq[j] = q[j] - ld3(x_tilde, d + j);
        }
        const float* M = mass16 + 16 * (size_t)bi;
        const float c = (fixed[bi] ? 1.0f + dirichlet : 1.0f) * h2inv;
        float H[4][4][9];  // block (i, j), column-major 3 x 3
        v3 G[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            v3 g = mk3(0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float m = M[4 * i + j];
                g = mk3(g.x + m * dq[j].x, g.y + m * dq[j].y, g.z + m * dq[j].z);
                const float hm = c * m;
#pragma unroll
                for (int k = 0; k < 9; ++k) H[i][j][k] = (k % 4 == 0) ? hm : 0.0f;
            }
            G[i] = c * g;
        }
        const float s4 = 4.0f * (kappa[bi] * volume[bi]);
        const v3 A[3] = {q[1], q[2], q[3]};
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
            v3 og = neg3(A[ii]);
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) og = og + dot3(A[ii], A[jj]) * A[jj];
            G[1 + ii] = G[1 + ii] + s4 * og;
        }
#pragma unroll
        for (int ii = 0; ii < 3; ++ii)
#pragma unroll
            for (int jj = ii; jj < 3; ++jj) {
                const float ai[3] = {A[ii].x, A[ii].y, A[ii].z}, aj[3] = {A[jj].x, A[jj].y, A[jj].z};
                float h[9];
                if (ii == jj) {
                    const float dd = dot3(A[ii], A[ii]) - 1.0f;
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                        for (int r = 0; r < 3; ++r) {
                            float e = ai[r] * ai[cc] + (r == cc ? dd : 0.0f);
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                const float ak[3] = {A[k].x, A[k].y, A[k].z};
                                e = e + ak[r] * ak[cc];
                            }
                            h[3 * cc + r] = e;
                        }
                } else {
                    const float dd = dot3(A[ii], A[jj]);
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                        for (int r = 0; r < 3; ++r) h[3 * cc + r] = aj[r] * ai[cc] + (r == cc ? dd : 0.0f);
                }
#pragma unroll
                for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                    for (int r = 0; r < 3; ++r) {
                        H[1 + ii][1 + jj][3 * cc + r] = H[1 + ii][1 + jj][3 * cc + r] + s4 * h[3 * cc + r];
                        if (ii != jj)
                            H[1 + jj][1 + ii][3 * r + cc] = H[1 + jj][1 + ii][3 * r + cc] + s4 * h[3 * cc + r];
                    }
            }
        int t = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            b[d + i] = make_float4(-G[i].x, -G[i].y, -G[i].z, 0.0f);
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
                diag[3 * (size_t)(d + i) + cc] = make_float4(H[i][i][3 * cc], H[i][i][3 * cc + 1], H[i][i][3 * cc + 2], 0.0f);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (i == j) continue;
                float* O = mat_val + slots[12 * (size_t)bi + t];
#pragma unroll
                for (int k = 0; k < 9; ++k) O[cs * k] = H[i][j][k];
                ++t;
            }
        }
    }
}

// fn_evaluate_abd_ground_collision (newton_solver.cpp:1333-1410): the floor barrier of a rigid mesh
// vertex, added to its body's DOF slots with weights (1, x_bar)
__global__ void k_abd_floor(uint32_t n, AbdDev abd, const uint8_t* __restrict__ pinned, const float4* __restrict__ x,
                            float floor_y, float kappa, const float* __restrict__ vert_area,
                            const float* __restrict__ dhat, const float* __restrict__ offset, float4* b, float4* diag,
                            const uint32_t* __restrict__ slots, uint32_t cs, float* mat_val)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!is_rigid(abd, i) || (pinned && pinned[i])) continue;
        const float dh = dhat[i], th = offset[i], dist = x[i].y - floor_y;
        if (!(dist - th < dh)) continue;
        const float stiff = kappa * vert_area[i];
        const float dd = dist - th;
        const float k1 = stiff * ((dh - dd) * (2.0f * logf(dd / dh) - dh / dd + 1.0f));
        const float qq = dh / dd;
        const float k2 = stiff * ((qq + 2.0f) * qq - 2.0f * logf(dd / dh) - 3.0f);
        const uint32_t bi = abd.body[i], d = abd.body_dof[bi];
        const float4 m = abd.model_x[i];
        const float w[4] = {1.0f, m.x, m.y, m.z};
        int t = 0;
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) {
            atomicAdd(&b[d + ii].y, -(w[ii] * k1));
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const float hv = w[ii] * w[jj] * k2;  // only the (y, y) entry of n n^T
                if (ii == jj) {
                    atomicAdd(&diag[3 * (size_t)(d + ii) + 1].y, hv);
                } else {
                    atomicAdd(mat_val + slots[12 * (size_t)bi + t] + cs * 4, hv);
                    ++t;
                }
            }
        }
    }
}

// after the solve: the rigid mesh vertices' increment J(x_bar) dq, so that the CCD bound, the line
// search and the small-step test see them move
__global__ void k_abd_expand(uint32_t n, AbdDev abd, float4* dx)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!is_rigid(abd, i)) continue;
        const uint32_t d = abd.body_dof[abd.body[i]];
        const v3 r = affine_apply(ld3(dx, d), ld3(dx, d + 1), ld3(dx, d + 2), ld3(dx, d + 3), abd.model_x[i]);
        dx[i] = make_float4(r.x, r.y, r.z, 0.0f);
    }
}

// one 16-byte vector atomic (sm_90 and later) per vertex record
__device__ __forceinline__ void red4(float4* p, float x, float y, float z) { atomicAdd(p, make_float4(x, y, z, 0.0f)); }

// adds the 3x3 block K (column-major [3 c + r]) into a diagonal record (three float4 columns)
__device__ __forceinline__ void red_diag(float4* D, const float* K)
{
#pragma unroll
    for (int c = 0; c < 3; ++c) red4(D + c, K[3 * c], K[3 * c + 1], K[3 * c + 2]);
}
// adds K (or its transpose) into an off-diagonal block whose component 3 c + r sits at O[cs (3 c + r)]
__device__ __forceinline__ void red_off(float* O, uint32_t cs, const float* K, bool t)
{
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) atomicAdd(O + cs * (3 * c + r), t ? K[3 * r + c] : K[3 * c + r]);
}

// fn_evaluate_stretch_face + fn_material_energy_assembly_stretch_face (newton_solver.cpp:1052-1100,
// 705-789): Baraff-Witkin stretch and shear added straight into b, the diagonal and the material
// blocks; slots: the 6 off-diagonal blocks (0,1) (0,2) (1,0) (1,2) (2,0) (2,1) of each face
__global__ void k_stretch_bw98(uint32_t nf, const uint4* __restrict__ faces, const float4* __restrict__ dm,
                               const float* __restrict__ area, const float2* __restrict__ ml, float mu, float lambda,
                               const float4* __restrict__ x, float4* b, float4* diag, const uint32_t* __restrict__ slots,
                               uint32_t cs, float* mat_val)
{
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        const uint4 fc = faces[f];
        const float2 m = ml ? ml[f] : make_float2(mu, lambda);
        Bw98Out o;
        bw98_face(ld3(x, fc.x), ld3(x, fc.y), ld3(x, fc.z), dm[f], m.x, m.y, area[f], o);
        const uint32_t v[3] = {fc.x, fc.y, fc.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            red4(&b[v[a]], -o.g[a].x, -o.g[a].y, -o.g[a].z);
            red_diag(diag + 3 * (size_t)v[a], o.K[a]);
        }
        const uint32_t* sl = slots + 6 * (size_t)f;
        red_off(mat_val + sl[0], cs, o.K[3], false);  // (0,1)
        red_off(mat_val + sl[1], cs, o.K[4], false);  // (0,2)
        red_off(mat_val + sl[2], cs, o.K[3], true);   // (1,0)
        red_off(mat_val + sl[3], cs, o.K[5], false);  // (1,2)
        red_off(mat_val + sl[4], cs, o.K[4], true);   // (2,0)
        red_off(mat_val + sl[5], cs, o.K[5], true);   // (2,1)
    }
}

// fn_evaluate_bending + fn_material_energy_assembly_bending (newton_solver.cpp:1102-1175, 790-801):
// dihedral-angle bending, Gauss-Newton blocks k g_i g_j^T; slots as k_bending
__global__ void k_bending_dihedral(uint32_t nb, const uint4* __restrict__ stencil, const float* __restrict__ rest_angle,
                                   const float* __restrict__ hbar, const float* __restrict__ kper, float k,
                                   float scaling, const float4* __restrict__ x, float4* b, float4* diag,
                                   const uint32_t* __restrict__ slots, uint32_t cs, float* mat_val)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nb; s += gridDim.x * blockDim.x) {
        const uint4 e = stencil[s];
        const uint32_t v[4] = {e.x, e.y, e.z, e.w};
        v3 g[4];
        const float theta = dihedral_angle_grad(ld3(x, e.x), ld3(x, e.y), ld3(x, e.z), ld3(x, e.w), g);
        const float stiff = ((kper ? kper[s] : k) * scaling) * hbar[s];
        const float sd = stiff * (theta - rest_angle[s]);
        int t = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            red4(&b[v[i]], -(sd * g[i].x), -(sd * g[i].y), -(sd * g[i].z));
            const float gi[3] = {g[i].x, g[i].y, g[i].z};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float gj[3] = {g[j].x, g[j].y, g[j].z};
                float K[9];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < 3; ++r) K[3 * c + r] = stiff * (gi[r] * gj[c]);
                if (i == j) {
                    red_diag(diag + 3 * (size_t)v[i], K);
                } else {
                    red_off(mat_val + slots[12 * (size_t)s + t], cs, K, false);
                    ++t;
                }
            }
        }
    }
}

// ---- deterministic assembly (LCS_NEWTON_DETERMINISTIC)
// The producers above, split in two: each element writes its terms (gradient, Hessian blocks) to its own
// slots of `el`, then every row and every material block sums its elements' terms in element order.  The
// terms are computed by the same expressions as above and each sum adds them one at a time onto the same
// start value (the inertia term for b and the diagonal, zero for a block), so only the order of the
// additions is fixed.  Per element: spring 12 floats (gradient of end 0, then the Hessian block), face 64
// (the three corner gradients, then the blocks (0,0) (1,1) (2,2) (0,1) (0,2) (1,2)), stencil 16 (dihedral:
// the four gradients, stiffness, stiffness x angle defect; quadratic: the four gradients).
__global__ void k_springs_det(uint32_t ne, const uint2* __restrict__ edges, const float* __restrict__ rest_len,
                              const float* __restrict__ kper, float k_scalar, const float4* __restrict__ x,
                              float* __restrict__ el)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const float k = kper ? kper[e] : k_scalar;
        const uint2 ed = edges[e];
        const float4 p0 = x[ed.x], p1 = x[ed.y];
        const float dx = p0.x - p1.x, dy = p0.y - p1.y, dz = p0.z - p1.z;
        const float l = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1.19209290E-7f);
        const float L = rest_len[e];
        const float C = l - L;
        const float il = 1.0f / l, il2 = il * il;
        float* o = el + 12 * (size_t)e;
        o[0] = k * dx * il * C;
        o[1] = k * dy * il * C;
        o[2] = k * dz * il * C;
        const float a = k * il2, c = k * fmaxf(1.0f - L * il, 0.0f);
        const float d[3] = {dx, dy, dz};
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int r = 0; r < 3; ++r) o[3 + 3 * cc + r] = a * d[r] * d[cc] + c * ((r == cc ? 1.0f : 0.0f) - il2 * d[r] * d[cc]);
    }
}

__global__ void k_stretch_bw98_det(uint32_t nf, const uint4* __restrict__ faces, const float4* __restrict__ dm,
                                   const float* __restrict__ area, const float2* __restrict__ ml, float mu,
                                   float lambda, const float4* __restrict__ x, float* __restrict__ el)
{
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        const uint4 fc = faces[f];
        const float2 m = ml ? ml[f] : make_float2(mu, lambda);
        Bw98Out o;
        bw98_face(ld3(x, fc.x), ld3(x, fc.y), ld3(x, fc.z), dm[f], m.x, m.y, area[f], o);
        float* q = el + 64 * (size_t)f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            q[3 * a] = o.g[a].x;
            q[3 * a + 1] = o.g[a].y;
            q[3 * a + 2] = o.g[a].z;
        }
#pragma unroll
        for (int b = 0; b < 6; ++b)
#pragma unroll
            for (int c = 0; c < 9; ++c) q[9 + 9 * b + c] = o.K[b][c];
    }
}

__global__ void k_bending_dihedral_det(uint32_t nb, const uint4* __restrict__ stencil, const float* __restrict__ rest_angle,
                                       const float* __restrict__ hbar, const float* __restrict__ kper, float k,
                                       float scaling, const float4* __restrict__ x, float* __restrict__ el)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nb; s += gridDim.x * blockDim.x) {
        const uint4 e = stencil[s];
        v3 g[4];
        const float theta = dihedral_angle_grad(ld3(x, e.x), ld3(x, e.y), ld3(x, e.z), ld3(x, e.w), g);
        const float stiff = ((kper ? kper[s] : k) * scaling) * hbar[s];
        float* q = el + 16 * (size_t)s;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            q[3 * i] = g[i].x;
            q[3 * i + 1] = g[i].y;
            q[3 * i + 2] = g[i].z;
        }
        q[12] = stiff;
        q[13] = stiff * (theta - rest_angle[s]);
    }
}

__global__ void k_bending_det(uint32_t nb, const uint4* __restrict__ stencil, const float* __restrict__ Q, float k,
                              const float4* __restrict__ x, const float4* __restrict__ rest, float* __restrict__ el)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nb; s += gridDim.x * blockDim.x) {
        const uint4 st = stencil[s];
        const uint32_t v[4] = {st.x, st.y, st.z, st.w};
        float3 u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float4 p = x[v[j]], r = rest[v[j]];
            u[j] = make_float3(p.x - r.x, p.y - r.y, p.z - r.z);
        }
        const float* qq = Q + 16 * (size_t)s;
        float* o = el + 16 * (size_t)s;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float3 g = make_float3(0.f, 0.f, 0.f);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float qij = k * qq[4 * i + j];
                g.x += qij * u[j].x;
                g.y += qij * u[j].y;
                g.z += qij * u[j].z;
            }
            o[3 * i] = g.x;
            o[3 * i + 1] = g.y;
            o[3 * i + 2] = g.z;
        }
    }
}

// local pair t of a stencil's 12 ordered pairs (i, j), i != j, in the producers' loop order
__device__ __forceinline__ void stencil_pair(uint32_t t, int& i, int& j)
{
    i = (int)(t / 3);
    const int jj = (int)(t % 3);
    j = jj < i ? jj : jj + 1;
}

struct DetEl {
    const float* el;
    size_t off_face, off_bend;
    const float* Q;  // quadratic bending
    float k_quad;
};

// b and the diagonal of each row: the inertia term already there, then its elements' terms in element order
__global__ void k_det_rows(uint32_t n, const uint32_t* __restrict__ vptr, const uint2* __restrict__ vent, DetEl D,
                           float4* __restrict__ b, float4* __restrict__ diag)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        float4 bv = b[v];
        float4 dc[3] = {diag[3 * (size_t)v], diag[3 * (size_t)v + 1], diag[3 * (size_t)v + 2]};
        auto add_block = [&](const float* K) {  // column-major [3 c + r]
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                dc[c].x += K[3 * c];
                dc[c].y += K[3 * c + 1];
                dc[c].z += K[3 * c + 2];
            }
        };
        const uint32_t e1 = vptr[v + 1];
        for (uint32_t q = vptr[v]; q < e1; ++q) {
            const uint2 en = vent[q];
            const uint32_t kind = en.y >> 4, a = en.y & 15u;
            if (kind == 0) {  // spring: end 0 takes -g, end 1 +g; both the block
                const float* o = D.el + 12 * (size_t)en.x;
                if (a == 0) { bv.x += -o[0]; bv.y += -o[1]; bv.z += -o[2]; }
                else { bv.x += o[0]; bv.y += o[1]; bv.z += o[2]; }
                add_block(o + 3);
            } else if (kind == 1) {  // face corner a
                const float* o = D.el + D.off_face + 64 * (size_t)en.x;
                bv.x += -o[3 * a]; bv.y += -o[3 * a + 1]; bv.z += -o[3 * a + 2];
                add_block(o + 9 + 9 * a);
            } else if (kind == 2) {  // dihedral stencil vertex a: -sd g_a, block stiff g_a g_a^T
                const float* o = D.el + D.off_bend + 16 * (size_t)en.x;
                const float stiff = o[12], sd = o[13];
                const float gi[3] = {o[3 * a], o[3 * a + 1], o[3 * a + 2]};
                bv.x += -(sd * gi[0]); bv.y += -(sd * gi[1]); bv.z += -(sd * gi[2]);
                float K[9];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < 3; ++r) K[3 * c + r] = stiff * (gi[r] * gi[c]);
                add_block(K);
            } else {  // quadratic stencil vertex a: -g_a, block k Q_aa I
                const float* o = D.el + D.off_bend + 16 * (size_t)en.x;
                bv.x += -o[3 * a]; bv.y += -o[3 * a + 1]; bv.z += -o[3 * a + 2];
                const float qaa = D.k_quad * D.Q[16 * (size_t)en.x + 5 * a];
                dc[0].x += qaa;
                dc[1].y += qaa;
                dc[2].z += qaa;
            }
        }
        b[v] = bv;
        diag[3 * (size_t)v] = dc[0];
        diag[3 * (size_t)v + 1] = dc[1];
        diag[3 * (size_t)v + 2] = dc[2];
    }
}

// each material block from zero: its elements' blocks in element order, written at its base (components cs apart)
__global__ void k_det_blocks(uint32_t nblk, const uint32_t* __restrict__ bptr, const uint2* __restrict__ bent,
                             const uint32_t* __restrict__ bbase, DetEl D, uint32_t cs, float* __restrict__ mat_val)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nblk; j += gridDim.x * blockDim.x) {
        float acc[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) acc[q] = 0.0f;
        const uint32_t e1 = bptr[j + 1];
        for (uint32_t q = bptr[j]; q < e1; ++q) {
            const uint2 en = bent[q];
            const uint32_t kind = en.y >> 4, t = en.y & 15u;
            if (kind == 0) {  // spring: -H in both directions
                const float* H = D.el + 12 * (size_t)en.x + 3;
#pragma unroll
                for (int c = 0; c < 9; ++c) acc[c] += -H[c];
            } else if (kind == 1) {  // face pair t: (0,1) (0,2) (1,0) (1,2) (2,0) (2,1) from blocks 3, 4, 3^T, 5, 4^T, 5^T
                const float* o = D.el + D.off_face + 64 * (size_t)en.x;
                const int m = t == 0 || t == 2 ? 3 : t == 1 || t == 4 ? 4 : 5;
                const bool tr = t == 2 || t == 4 || t == 5;
                const float* K = o + 9 + 9 * m;
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < 3; ++r) acc[3 * c + r] += tr ? K[3 * r + c] : K[3 * c + r];
            } else if (kind == 2) {  // dihedral pair (i, j): stiff g_i g_j^T
                const float* o = D.el + D.off_bend + 16 * (size_t)en.x;
                int i, jj;
                stencil_pair(t, i, jj);
                const float stiff = o[12];
                const float gi[3] = {o[3 * i], o[3 * i + 1], o[3 * i + 2]};
                const float gj[3] = {o[3 * jj], o[3 * jj + 1], o[3 * jj + 2]};
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < 3; ++r) acc[3 * c + r] += stiff * (gi[r] * gj[c]);
            } else {  // quadratic pair (i, j): k Q_ij I
                int i, jj;
                stencil_pair(t, i, jj);
                const float qij = D.k_quad * D.Q[16 * (size_t)en.x + 4 * i + jj];
                acc[0] += qij;
                acc[4] += qij;
                acc[8] += qij;
            }
        }
        float* O = mat_val + bbase[j];
#pragma unroll
        for (int c = 0; c < 9; ++c) O[(size_t)cs * c] = acc[c];
    }
}

// Contact pairs in a canonical order: by (type, v0, v1) after (v2, v3), 21 bits per vertex index.
// keys_lo: pass 1 (v2, v3); pass 2 re-keys the pass-1 order by (type, v0, v1) and sorts stably.
__global__ void k_pair_keys(const lcs_pair* __restrict__ pairs, const uint32_t* d_count, uint32_t cap, int hi,
                            const uint32_t* __restrict__ order, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                            uint32_t* d_n)
{
    const uint32_t n = pair_count(d_count, cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_n = n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t p = order ? order[k] : k;
        const PairView P = load_pair(pairs, p);
        keys[k] = hi ? ((uint64_t)P.type << 42) | ((uint64_t)P.v[0] << 21) | (uint64_t)P.v[1]
                     : ((uint64_t)P.v[2] << 21) | (uint64_t)P.v[3];
        vals[k] = p;
    }
}

__global__ void k_pair_gather(const lcs_pair* __restrict__ pairs, const uint32_t* d_n, const uint32_t* __restrict__ order,
                              lcs_pair* __restrict__ out)
{
    const uint32_t n = *d_n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) out[k] = pairs[order[k]];
}

// row keys of the contact gradient / diagonal terms: 4 per pair (vertex i), pairs without contact last
__global__ void k_cg_keys(const lcs_pair* __restrict__ pairs, const uint32_t* d_n, uint32_t n_rows,
                          uint64_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t* d_n4)
{
    const uint32_t n = *d_n;
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_n4 = 4 * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const PairView P = load_pair(pairs, k);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            keys[4 * (size_t)k + i] = P.type ? P.v[i] : n_rows;
            vals[4 * (size_t)k + i] = 4u * k + (uint32_t)i;
        }
    }
}

// each row's contact gradient and diagonal block (k_grad_diag's terms), summed in canonical pair order and
// added once; one thread per row segment
__global__ void k_cg_rows(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals, const uint32_t* d_n4,
                          uint32_t n_rows, const lcs_pair* __restrict__ pairs, float4* __restrict__ b,
                          float4* __restrict__ diag)
{
    const uint32_t n = *d_n4;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint64_t key = keys[s];
        if (key >= n_rows || (s > 0 && keys[s - 1] == key)) continue;
        float g3[3] = {0.f, 0.f, 0.f}, h9[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) h9[q] = 0.0f;
        for (uint32_t t = s; t < n && keys[t] == key; ++t) {
            const uint32_t v = vals[t];
            const PairView P = load_pair(pairs, v >> 2);
            const float w = P.w[v & 3u];
            const float g = P.k1 * w;
            g3[0] += g * P.n.x;
            g3[1] += g * P.n.y;
            g3[2] += g * P.n.z;
            const float h = P.k2 * w * w;
            const float nn[3] = {P.n.x, P.n.y, P.n.z};
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r) h9[3 * c + r] += h * (nn[r] * nn[c]);
        }
        const uint32_t r = (uint32_t)key;
        float4 bv = b[r];
        bv.x += g3[0];
        bv.y += g3[1];
        bv.z += g3[2];
        b[r] = bv;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float4 d = diag[3 * (size_t)r + c];
            d.x += h9[3 * c];
            d.y += h9[3 * c + 1];
            d.z += h9[3 * c + 2];
            diag[3 * (size_t)r + c] = d;
        }
    }
}

// fn_apply_dx (newton_solver.cpp:491-503) with alpha = 1, and the |dx|_inf of the small-step test
__global__ void k_apply_unit(uint32_t n, const float4* __restrict__ x0, const float4* __restrict__ dx, float4* __restrict__ x,
                             Status* st, AbdDev abd)
{
    float m = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = stepped(abd, i, x0, dx, 1.0f);
        if (!is_rigid(abd, i)) {  // the solve's unknowns: soft vertices and DOF slots (sa_cgX)
            const float4 d = dx[i];
            m = fmaxf(m, sqrtf(d.x * d.x + d.y * d.y + d.z * d.z));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if (lane_id() == 0) atomic_max_pos(&st->max_dx, m);
}

// apply_final_dx with alpha = the CCD step bound, and the Dirichlet check (newton_solver.cpp:3741-3752, 3858-3882)
__global__ void k_apply_final(uint32_t n, const float4* __restrict__ x0, const float4* __restrict__ dx,
                              float4* __restrict__ x, const uint8_t* __restrict__ pinned,
                              const float4* __restrict__ x_tilde, Status* st, int use_ls_alpha, AbdDev abd)
{
    const float alpha = use_ls_alpha ? st->alpha : st->toi;
    float m = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 r = stepped(abd, i, x0, dx, alpha);
        x[i] = r;
        if (pinned && pinned[i]) {
            const float4 t = x_tilde[i];
            const float ex = r.x - t.x, ey = r.y - t.y, ez = r.z - t.z;
            m = fmaxf(m, sqrtf(ex * ex + ey * ey + ez * ez));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if (lane_id() == 0) atomic_max_pos(&st->dirichlet, m);
}

// fn_gound_collision_ccd, newton_solver.cpp:952-1000
__global__ void k_floor_ccd(uint32_t n, const float4* __restrict__ x0, const float4* __restrict__ x,
                            const float* __restrict__ offset, const uint8_t* __restrict__ pinned, float floor_y,
                            Status* st)
{
    float m = 1.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (pinned && pinned[i]) continue;
        const float off = offset[i], cy = x[i].y;
        if (cy - off < floor_y) {
            const float iy = x0[i].y;
            m = fminf(m, (iy - off - floor_y) / (iy - cy) / 1.25f);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if (lane_id() == 0 && m < 1.0f) atomicMin(reinterpret_cast<int*>(&st->toi), __float_as_int(fmaxf(m, 0.0f)));
}

// fn_update_velocity, newton_solver.cpp:606-633
__global__ void k_update_velocity(uint32_t n, float dt, float damping, const float4* __restrict__ x,
                                  const float4* __restrict__ x_step_start, float4* __restrict__ v)
{
    const float f = expf(-damping * dt);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = x_step_start[i], c = x[i];
        v[i] = make_float4((c.x - a.x) / dt * f, (c.y - a.y) / dt * f, (c.z - a.z) / dt * f, 0.0f);
    }
}

__global__ void k_copy4(uint32_t n, const float4* __restrict__ a, float4* __restrict__ b)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

__global__ void k_save_ccd_counts(const Status* st, uint32_t* prev)
{
    prev[0] = st->cnt[3];
    prev[1] = st->cnt[4];
}

__global__ void k_pcg_to_status(const lcs_pcg_stats* ps, Status* st)
{
    st->pcg_iters = ps->iterations;
    st->pcg_rel = ps->rel_residual;
    st->pcg_status = ps->status;
}

// ---- energy line search (line_search with use_energy_linesearch, newton_solver.cpp:3790-3834)
// The reference evaluates the energy at alpha = 0 and then at toi, toi / 2, ... one step length at
// a time with a host round trip each, and takes the first with E < E(0) + Epsilon; a step length
// below 1e-4 is an error.  Here one launch evaluates E at alpha = 0 and at kLsSlots - 1 successive
// halvings together (every element loads its vertices once), and a one-thread kernel picks the
// step on the device, so the usual case costs no host synchronisation.
constexpr int kLsSlots = 8;

struct LsArgs {
    uint32_t V, E, Fs, B, P;  // vertices, springs, stretch faces, bending stencils, pair capacity
    const float4 *x0, *dx, *xt, *rest;
    const float* mass;
    const uint8_t* pinned;
    float h2inv, dirichlet;
    const uint2* edges;
    const float* rest_len;
    float spring_k;
    const float* spring_kper;
    const float2* ml;
    const float* bend_kper;
    float bend_scaling;
    const uint4* sfaces;
    const float4* dm;
    const float* sarea;
    float mu, lambda;
    const uint4* bend;
    const float *rest_angle, *hbar, *Q;
    float kb;         // dihedral: bending_k * scaling; quadratic: bending_k
    int bending_model;
    const lcs_pair* pairs;
    const uint32_t* pair_count;
    const float *dhat, *offset;
    AbdDev abd;
    uint32_t NB;
    const float *bmass, *bvol, *bkappa;
};

__device__ __forceinline__ float ls_alpha(float toi, int j)
{
    float a = toi;
    for (int k = 0; k < j; ++k) a /= 2.0f;
    return a;
}

__device__ __forceinline__ v3 ls_pos(const LsArgs& a, uint32_t v, float alpha)
{
    const float4 p = a.x0[v], d = a.dx[v];
    return mk3(p.x + alpha * d.x, p.y + alpha * d.y, p.z + alpha * d.z);
}

// E(alpha_k) for slot 0 (alpha = 0) and slots k >= 1 (alpha = toi / 2^(j0 + k - 1)): inertia with the
// Dirichlet factor, the stretch and bending models, and the barrier energy of the iteration-start pairs
// (fn_calc_energy_*, solver_interface.cpp:505-728; compute_contact_energy_from_iter_start_list)
template <int NS>
__global__ void __launch_bounds__(256) k_ls_energy(LsArgs a, int j0, const Status* __restrict__ st, double* E)
{
    const uint32_t npairs = a.P ? pair_count(a.pair_count, a.P) : 0;
    const uint32_t n = max(max(max(a.V, a.E), max(a.Fs, a.B)), max(npairs, a.NB));
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n_round = (n + stride - 1) / stride * stride;
    const float toi = st->toi;
    float al[NS];
    al[0] = 0.0f;
#pragma unroll
    for (int k = 1; k < NS; ++k) al[k] = ls_alpha(toi, j0 + k - 1);
    double e[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) e[k] = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += stride) {
        if (i < a.V && !(a.abd.body && a.abd.body[i] != kInvalid)) {  // bodies: the per-body terms below
            const float4 t = a.xt[i];
            const float m = a.mass[i];
            const bool fixed = a.pinned && a.pinned[i];
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                const v3 d = ls_pos(a, i, al[k]) - mk3(t.x, t.y, t.z);
                float en = a.h2inv * dot3(d, d) * m / 2.0f;
                if (fixed) en = a.dirichlet * en;
                e[k] += (double)en;
            }
        }
        if (i < a.E) {
            const uint2 ed = a.edges[i];
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                const v3 d = ls_pos(a, ed.y, al[k]) - ls_pos(a, ed.x, al[k]);
                const float C = sqrtf(dot3(d, d)) - a.rest_len[i];
                e[k] += (double)(0.5f * (a.spring_kper ? a.spring_kper[i] : a.spring_k) * C * C);
            }
        }
        if (i < a.Fs) {
            const uint4 fc = a.sfaces[i];
            const float4 dm = a.dm[i];
            const float ar = a.sarea[i];
            const float2 ml = a.ml ? a.ml[i] : make_float2(a.mu, a.lambda);
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                const v3 x0 = ls_pos(a, fc.x, al[k]), e1 = ls_pos(a, fc.y, al[k]) - x0, e2 = ls_pos(a, fc.z, al[k]) - x0;
                const v3 Fu = mk3(__fmaf_rn(e2.x, dm.y, e1.x * dm.x), __fmaf_rn(e2.y, dm.y, e1.y * dm.x),
                                  __fmaf_rn(e2.z, dm.y, e1.z * dm.x));
                const v3 Fv = mk3(__fmaf_rn(e2.x, dm.w, e1.x * dm.z), __fmaf_rn(e2.y, dm.w, e1.y * dm.z),
                                  __fmaf_rn(e2.z, dm.w, e1.z * dm.z));
                const float su = sqrtf(dot3(Fu, Fu)) - 1.0f, sv = sqrtf(dot3(Fv, Fv)) - 1.0f, i6 = dot3(Fu, Fv);
                e[k] += (double)(ar * (0.5f * ml.x * (su * su + sv * sv) + 0.5f * ml.y * (i6 * i6)));
            }
        }
        if (i < a.B) {
            const uint4 st4 = a.bend[i];
            const uint32_t v[4] = {st4.x, st4.y, st4.z, st4.w};
            if (a.bending_model == LCS_BENDING_DIHEDRAL) {
                const float kb = a.bend_kper ? a.bend_kper[i] : a.kb, hb = a.hbar[i];
                const float ra = a.rest_angle[i];
#pragma unroll
                for (int k = 0; k < NS; ++k) {
                    v3 g[4];
                    const float d = dihedral_angle_grad(ls_pos(a, v[0], al[k]), ls_pos(a, v[1], al[k]),
                                                        ls_pos(a, v[2], al[k]), ls_pos(a, v[3], al[k]), g) - ra;
                    e[k] += (double)(0.5f * kb * a.bend_scaling * hb * d * d);
                }
            } else {  // quadratic: E = k/2 sum_ij Q_ij (x_i - X_i).(x_j - X_j)
                const float* q = a.Q + 16 * (size_t)i;
#pragma unroll 1
                for (int k = 0; k < NS; ++k) {
                    v3 u[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float4 r = a.rest[v[j]];
                        u[j] = ls_pos(a, v[j], al[k]) - mk3(r.x, r.y, r.z);
                    }
                    float en = 0.0f;
#pragma unroll
                    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
                        for (int jj = 0; jj < 4; ++jj) en += q[4 * ii + jj] * dot3(u[ii], u[jj]);
                    e[k] += (double)(0.5f * a.kb * en);
                }
            }
        }
        if (i < a.NB) {  // fn_calc_energy_abd_inertia / _abd_ortho (solver_interface.cpp:631-728)
            const uint32_t d = a.abd.body_dof[i];
            const float* M = a.bmass + 16 * (size_t)i;
            const bool fixed = a.abd.fixed[i] != 0;
            const float kv = a.bkappa[i] * a.bvol[i];
#pragma unroll 1
            for (int k = 0; k < NS; ++k) {
                v3 q[4], dq[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    q[j] = ls_pos(a, d + j, al[k]);
                    const float4 t = a.xt[d + j];
                    dq[j] = q[j] - mk3(t.x, t.y, t.z);
                }
                float ei = 0.0f;
#pragma unroll
                for (int ii = 0; ii < 4; ++ii)
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj) ei += a.h2inv * dot3(dq[ii], dq[jj]) * M[4 * ii + jj] / 2.0f;
                if (fixed) ei = a.dirichlet * ei;
                float eo = 0.0f;
#pragma unroll
                for (int ii = 0; ii < 3; ++ii)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) {
                        const float tt = dot3(q[1 + ii], q[1 + jj]) - (ii == jj ? 1.0f : 0.0f);
                        eo += tt * tt;
                    }
                e[k] += (double)ei + (double)(eo * kv);
            }
        }
        if (i < npairs) {
            const PairView P = load_pair(a.pairs, i);
            if (P.type) {
                const float dh = 0.5f * (a.dhat[P.v[0]] + a.dhat[P.v[2]]);
                const float th = a.offset[P.v[0]] + a.offset[P.v[2]];
#pragma unroll
                for (int k = 0; k < NS; ++k) {
                    const v3 diff = ((P.w[0] * ls_pos(a, P.v[0], al[k]) + P.w[1] * ls_pos(a, P.v[1], al[k])) +
                                     P.w[2] * ls_pos(a, P.v[2], al[k])) + P.w[3] * ls_pos(a, P.v[3], al[k]);
                    const float d = sqrtf(dot3(diff, diff));
                    if (d < th + dh) e[k] += (double)(P.stiff * barrier_e(d - th, dh));
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        double v = e[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        if (lane_id() == 0 && v != 0.0) atomicAdd(E + k, v);
    }
}

// the first slot k >= 1 with E_k < E_0 + Epsilon (newton_solver.cpp:3810-3834); small steps skip the
// search (newton_solver.cpp:3774-3788); step lengths below 1e-4 are a failure
__global__ void k_ls_pick(const double* __restrict__ E, int j0, float small_step, Status* st)
{
    const float toi = st->toi;
    st->dirichlet = 0.0f;  // the apply that follows measures it again
    if (st->max_dx < small_step) {
        st->alpha = toi;
        st->ls_iters = 0;
        st->ls_state = 1;
        return;
    }
    const double limit = E[0] + (double)1.19209290E-7f;
    for (int k = 1; k < kLsSlots; ++k) {
        const int j = j0 + k - 1;
        const float alpha = ls_alpha(toi, j);
        if (j > 0 && alpha < 1e-4f) {
            st->alpha = alpha;
            st->ls_iters = j;
            st->ls_state = 3;
            return;
        }
        if (E[k] < limit) {
            st->alpha = alpha;
            st->ls_iters = j;
            st->ls_state = 1;
            return;
        }
    }
    st->alpha = ls_alpha(toi, j0 + kLsSlots - 2);
    st->ls_iters = j0 + kLsSlots - 2;
    st->ls_state = 2;
}

// ---- batched scenes: per-scene step bound, small-step and Dirichlet tests
__global__ void k_b_reset(uint32_t S, float* bsc)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        bsc[s] = 1.0f;          // toi
        bsc[S + s] = 0.0f;      // max |dx|
        bsc[2 * S + s] = 0.0f;  // Dirichlet error
    }
}

// lane-aggregated max into per-scene slots (vertices of a warp usually share a scene)
__device__ __forceinline__ void scene_max(float* slots, uint32_t s, float m)
{
    const uint32_t mask = __activemask();
    if (mask == 0xFFFFFFFFu) {  // the same for every lane of the warp
        const uint32_t s0 = __shfl_sync(mask, s, 0);
        if (__all_sync(mask, s == s0)) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(mask, m, o));
            if (lane_id() == 0 && m > 0.0f) atomic_max_pos(slots + s, m);
            return;
        }
    }
    if (m > 0.0f) atomic_max_pos(slots + s, m);
}

__global__ void k_b_apply_unit(uint32_t n, const uint32_t* __restrict__ vscene, uint32_t S,
                               const float4* __restrict__ x0, const float4* __restrict__ dx, float4* __restrict__ x,
                               float* bsc, AbdDev abd)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = stepped(abd, i, x0, dx, 1.0f);
        const float4 d = dx[i];
        scene_max(bsc + S, vscene[i], is_rigid(abd, i) ? 0.0f : sqrtf(d.x * d.x + d.y * d.y + d.z * d.z));
    }
}

__global__ void k_b_apply_final(uint32_t n, const uint32_t* __restrict__ vscene, uint32_t S,
                                const float4* __restrict__ x0, const float4* __restrict__ dx, float4* __restrict__ x,
                                const uint8_t* __restrict__ pinned, const float4* __restrict__ x_tilde, float* bsc,
                                AbdDev abd)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = vscene[i];
        const float alpha = bsc[s];
        const float4 r = stepped(abd, i, x0, dx, alpha);
        x[i] = r;
        float m = 0.0f;
        if (pinned && pinned[i]) {
            const float4 t = x_tilde[i];
            const float ex = r.x - t.x, ey = r.y - t.y, ez = r.z - t.z;
            m = sqrtf(ex * ex + ey * ey + ez * ez);
        }
        scene_max(bsc + 2 * S, s, m);
    }
}

template <typename T>
cudaError_t dalloc(T*& p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (count ? count : 1));
}

template <typename T>
cudaError_t upload(T*& p, const T* host, size_t count)
{
    cudaError_t e = dalloc(p, count);
    if (e == cudaSuccess && host && count) e = cudaMemcpy(p, host, sizeof(T) * count, cudaMemcpyHostToDevice);
    return e;
}

}  // namespace

enum { kPhBuild, kPhMaterial, kPhDcdBroad, kPhDcdNarrow, kPhAssembly, kPhPcg, kPhCcdBroad, kPhCcdNarrow, kPhApply, kPhases };

struct lcs_newton {
    lcs_scene_desc d{};
    int flags = 0;
    bool plain = false, fp64 = false, profile = false;
    uint32_t V = 0, F = 0, E = 0, B = 0;
    cudaStream_t s = nullptr;
    bool own_stream = false;
    // fused mode: the edge-tree lane of the broad phase runs on s2, forked from and joined back to s
    cudaStream_t s2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // fused mode: the material producers run on s3 beside the DCD broad and narrow phases
    cudaStream_t s3 = nullptr;
    cudaEvent_t fork_m = nullptr, join_m = nullptr;
    // mesh
    uint4* faces = nullptr;
    uint2* edges = nullptr;
    uint4* bend = nullptr;
    // affine bodies
    uint32_t NB = 0;
    uint32_t* body_dof = nullptr;
    float *bmass = nullptr, *bvol = nullptr, *bkappa = nullptr;
    uint8_t* bfixed = nullptr;
    float4* model_x = nullptr;
    int8_t* slot = nullptr;
    uint32_t* body_slots = nullptr;  // material-matrix slots of each body's 12 off-diagonal blocks
    float2* ml = nullptr;           // per-face mu, lambda (or null: the scalars)
    float *bend_kper = nullptr, *spring_kper = nullptr;  // per-stencil / per-edge stiffness (or null)
    uint4* sfaces = nullptr;        // BW98 stretch faces
    float4* dm = nullptr;           // their rest Dm^-1
    float *sarea = nullptr, *rest_angle = nullptr, *hbar = nullptr;
    uint32_t Fs = 0;
    float *Q = nullptr, *rest_len = nullptr, *vert_area = nullptr, *face_area = nullptr, *edge_area = nullptr;
    float *mass = nullptr, *dhat = nullptr, *offset = nullptr;
    uint32_t* body = nullptr;
    uint8_t* pinned = nullptr;
    int8_t* group = nullptr;
    Anim* anim = nullptr;
    float4 *rest = nullptr, *x = nullptr, *v = nullptr, *x_step = nullptr, *x_iter = nullptr, *x_tilde = nullptr;
    float4 *target = nullptr, *dx = nullptr, *b = nullptr, *diag = nullptr;
    // material BSR
    uint32_t nnz_mat = 0;
    uint32_t *mat_rp = nullptr, *mat_col = nullptr, *spring_slots = nullptr, *bend_slots = nullptr, *face_slots = nullptr;
    float* mat_val = nullptr;
    bool sell = false;             // material matrix in SELL-32 for the row-resident PCG (fused mode)
    // LCS_NEWTON_DETERMINISTIC: the cloth terms per element (det_el), then summed per row over the vertex's
    // elements (det_vptr / det_vent) and per material block over its elements (det_bptr / det_bent, written at
    // det_bbase), in element order; the contact pairs sorted into a canonical order and their gradient and
    // diagonal blocks summed per row in that order
    bool det = false;
    float* det_el = nullptr;
    size_t det_off_face = 0, det_off_bend = 0;  // float offsets of the face and stencil terms in det_el
    uint32_t det_nblk = 0;
    uint32_t *det_vptr = nullptr, *det_bptr = nullptr, *det_bbase = nullptr;
    uint2 *det_vent = nullptr, *det_bent = nullptr;  // (element, kind << 4 | local index)
    uint64_t *det_keys = nullptr, *det_keys_alt = nullptr;
    uint32_t *det_vals = nullptr, *det_vals_alt = nullptr, *det_hist = nullptr, *det_n = nullptr;
    lcs_pair* det_pairs = nullptr;  // the pairs in canonical order (scratch)
    uint32_t det_cap = 0;           // pairs the contact scratch holds
    bool cg1 = false;              // single-reduction row-resident PCG (two grid synchronisations per iteration)
    size_t sell_vals = 0;          // floats in mat_val
    uint32_t *sell_ptr = nullptr, *sell_col = nullptr;
    // the contact blocks rewritten as SELL-32 before each solve (fused single-scene mode)
    uint32_t *cs_width = nullptr, *cs_ptr = nullptr, *cs_col = nullptr;
    float* cs_val = nullptr;
    int* cs_ok = nullptr;
    uint32_t cs_cap = 0;  // slots
    // contact
    lcs_bvh *face_tree = nullptr, *edge_tree = nullptr;
    uint32_t cap_vf = 0, cap_ee = 0, cap_pairs = 0;
    uint32_t alloc_vf = 0, alloc_ee = 0, alloc_pairs = 0;  // capacities the buffers were allocated with
    uint2 *bp_vf = nullptr, *bp_ee = nullptr;
    // fused mode: DCD candidate lists (filled by traversal, or by filtering the previous iteration's
    // CCD lists, which hold every DCD candidate of the next iterate when that traversal ran to the end)
    uint2 *dcd_vf = nullptr, *dcd_ee = nullptr;
    uint32_t* prev_ccd = nullptr;  // device: the CCD candidate counts of the previous iteration
    bool filter_ok = false;
    bool carry_filter = false;     // the last CCD lists of the previous step describe the current positions
    bool full_traversal = false;   // LCS_NEWTON_FULL_TRAVERSAL
    bool ee_sym = false;           // every edge's first vertex: thickness 0, the same d_hat (ee_dhat)
    float ee_dhat = 0.0f;
    bool energy_ls = false;        // LCS_NEWTON_ENERGY_LINESEARCH
    bool global_matrix = false;    // LCS_NEWTON_PCG_GLOBAL_MATRIX
    double *ls_E = nullptr, *h_ls_E = nullptr;  // energies of one line-search round (device, pinned host)
    float* h_alpha = nullptr;      // pinned: the plain loop's chosen step length
    int32_t ls_halvings = 0;       // this step
    float last_alpha = 1.0f;
    lcs_pair* pairs = nullptr;
    lcs_assembler* asmb = nullptr;
    lcs_pcg* pcg = nullptr;
    Status *st = nullptr, *h_st = nullptr;
    float4 *h_x = nullptr, *h_v = nullptr, *h_x_iter = nullptr;  // pinned host mirrors (plain loop)
    // batched scenes (lcs_newton_create_batch): scene s owns vertices [voff[s], voff[s+1]) and
    // its faces/edges; trees are forests, step bounds, small-step tests and PCG are per scene
    bool batch = false;
    uint32_t S = 1;
    int cluster = 4;
    std::vector<uint32_t> h_voff, h_foff, h_eoff;
    uint32_t *vscene = nullptr, *voff_d = nullptr, *active = nullptr, *h_active = nullptr;
    uint8_t* rigid_scene_v = nullptr;  // batch with affine bodies: 1 for the vertices of scenes that hold one
    lcs_forest *face_forest = nullptr, *edge_forest = nullptr;
    float* bsc = nullptr;           // device: toi[S], max_dx[S], dirichlet[S]
    float* h_bsc = nullptr;         // pinned mirror
    lcs_pcg_stats *bpcg = nullptr, *h_bpcg = nullptr;
    std::vector<int32_t> sc_iters, sc_pcg;  // this step, per scene
    std::vector<lcs_newton_iter_record> iter_log;  // this step's Newton iterations (single scene)
    std::vector<float> sc_toi, sc_rel;
    std::vector<uint8_t> sc_done;
    // bookkeeping
    double time = 0.0;
    uint32_t frame = 0;
    int64_t total_newton = 0, total_pcg = 0;
    int32_t retries = 0;  // iterations re-run after growth, this step
    cudaEvent_t ev[kPhases + 1] = {};
    double phase_ms[kPhases] = {};
    int32_t phase_launch_count[kPhases] = {};
};

namespace {

AbdDev abd_of(const lcs_newton* h)
{
    return h->NB ? AbdDev{h->body, h->slot, h->model_x, h->body_dof, h->bfixed} : AbdDev{nullptr, nullptr, nullptr, nullptr, nullptr};
}

void free_contact(lcs_newton* h)
{
    if (h->bp_vf) cudaFree(h->bp_vf);
    if (h->bp_ee) cudaFree(h->bp_ee);
    if (h->dcd_vf) cudaFree(h->dcd_vf);
    if (h->dcd_ee) cudaFree(h->dcd_ee);
    if (h->pairs) cudaFree(h->pairs);
    if (h->asmb) lcs_assembler_destroy(h->asmb);
    for (void* q : {(void*)h->cs_width, (void*)h->cs_ptr, (void*)h->cs_col, (void*)h->cs_val, (void*)h->cs_ok})
        if (q) cudaFree(q);
    h->cs_width = h->cs_ptr = h->cs_col = nullptr;
    h->cs_val = nullptr;
    h->cs_ok = nullptr;
    h->cs_cap = 0;
    h->bp_vf = nullptr;
    h->bp_ee = nullptr;
    h->dcd_vf = nullptr;
    h->dcd_ee = nullptr;
    h->pairs = nullptr;
    h->asmb = nullptr;
    for (void* q : {(void*)h->det_keys, (void*)h->det_keys_alt, (void*)h->det_vals, (void*)h->det_vals_alt,
                    (void*)h->det_hist, (void*)h->det_pairs})
        if (q) cudaFree(q);
    h->det_keys = h->det_keys_alt = nullptr;
    h->det_vals = h->det_vals_alt = h->det_hist = nullptr;
    h->det_pairs = nullptr;
    h->det_cap = 0;
}

// (re)allocates the contact buffers whose capacity changed since they were allocated; the
// others keep their memory (resize_template grows one buffer at a time, narrow_phase.h:71-91)
int alloc_contact(lcs_newton* h)
{
    cudaError_t e = cudaSuccess;
    if (!h->bp_vf || h->alloc_vf != h->cap_vf) {
        if (h->bp_vf) cudaFree(h->bp_vf);
        if (h->dcd_vf) cudaFree(h->dcd_vf);
        h->bp_vf = nullptr;
        h->dcd_vf = nullptr;
        e = dalloc(h->bp_vf, h->cap_vf);
        if (e == cudaSuccess && !h->plain) e = dalloc(h->dcd_vf, h->cap_vf);
        h->alloc_vf = h->cap_vf;
    }
    if (e == cudaSuccess && (!h->bp_ee || h->alloc_ee != h->cap_ee)) {
        if (h->bp_ee) cudaFree(h->bp_ee);
        if (h->dcd_ee) cudaFree(h->dcd_ee);
        h->bp_ee = nullptr;
        h->dcd_ee = nullptr;
        e = dalloc(h->bp_ee, h->cap_ee);
        if (e == cudaSuccess && !h->plain) e = dalloc(h->dcd_ee, h->cap_ee);
        h->alloc_ee = h->cap_ee;
    }
    if (e == cudaSuccess && (!h->pairs || h->alloc_pairs != h->cap_pairs)) {
        if (h->pairs) cudaFree(h->pairs);
        if (h->asmb) lcs_assembler_destroy(h->asmb);
        h->pairs = nullptr;
        h->asmb = nullptr;
        e = dalloc(h->pairs, h->cap_pairs);
        h->alloc_pairs = h->cap_pairs;
        if (e == cudaSuccess && h->det) {  // canonical pair order: 4 row keys per pair for the gradient sums
            for (void* q : {(void*)h->det_keys, (void*)h->det_keys_alt, (void*)h->det_vals, (void*)h->det_vals_alt,
                            (void*)h->det_hist, (void*)h->det_pairs})
                if (q) cudaFree(q);
            const uint32_t kc = 4 * h->cap_pairs;
            h->det_keys = h->det_keys_alt = nullptr;
            h->det_vals = h->det_vals_alt = h->det_hist = nullptr;
            h->det_pairs = nullptr;
            e = dalloc(h->det_keys, kc);
            if (e == cudaSuccess) e = dalloc(h->det_keys_alt, kc);
            if (e == cudaSuccess) e = dalloc(h->det_vals, kc);
            if (e == cudaSuccess) e = dalloc(h->det_vals_alt, kc);
            if (e == cudaSuccess) e = dalloc(h->det_hist, rs::hist_words(kc));
            if (e == cudaSuccess) e = dalloc(h->det_pairs, h->cap_pairs);
            if (e == cudaSuccess && !h->det_n) e = dalloc(h->det_n, 2);
            h->det_cap = h->cap_pairs;
        }
        if (e == cudaSuccess && h->sell) {
            // SELL copy of the contact blocks: twice the assembler's block capacity plus a padded
            // group per slice; a step whose slices need more uses the CSR form
            for (void* q : {(void*)h->cs_col, (void*)h->cs_val})
                if (q) cudaFree(q);
            h->cs_col = nullptr;
            h->cs_val = nullptr;
            const uint64_t S = (h->V + 31) / 32;
            const uint64_t blocks = (uint64_t)(h->NB ? 56 : 12) * h->cap_pairs;
            h->cs_cap = (uint32_t)std::min<uint64_t>((2 * blocks + 31) / 32 + 4 * S, 0x7FFFFFFFu);
            if (!h->cs_width) e = dalloc(h->cs_width, S);
            if (e == cudaSuccess && !h->cs_ptr) e = dalloc(h->cs_ptr, S + 1);
            if (e == cudaSuccess && !h->cs_ok) e = dalloc(h->cs_ok, 1);
            if (e == cudaSuccess) e = dalloc(h->cs_col, 32ull * h->cs_cap);
            if (e == cudaSuccess) e = dalloc(h->cs_val, 288ull * h->cs_cap);
        }
        if (e == cudaSuccess)
            return h->NB ? lcs_assembler_create_abd(h->V, h->cap_pairs, &h->asmb)
                         : lcs_assembler_create(h->V, h->cap_pairs, &h->asmb);
    }
    return e == cudaSuccess ? LCS_OK : lcs_fail(LCS_ERR_CUDA, "lcs_newton: contact buffer allocation failed");
}

// runs f(begin, end) over [0, n) on the host's cores
template <typename F>
void parallel_ranges(size_t n, F f)
{
    unsigned t = std::thread::hardware_concurrency();
    t = t ? std::min(t, 32u) : 4u;
    if (n < 65536 || t == 1) {
        f((size_t)0, n);
        return;
    }
    std::vector<std::thread> pool;
    const size_t chunk = (n + t - 1) / t;
    for (unsigned k = 0; k < t; ++k) {
        const size_t b = k * chunk, e = std::min(n, b + chunk);
        if (b < e) pool.emplace_back(f, b, e);
    }
    for (auto& th : pool) th.join();
}

// material off-diagonal pattern from the element contributions; the slot of each contribution
// is its column's position in its sorted, de-duplicated row
int build_material_pattern(lcs_newton* h, const lcs_scene_desc* d)
{
    // contributions, in three ranges: spring k/2 (a->c, then c->a) when the stretch model is the
    // spring model; the ordered pairs (i, j), i != j, of each stretch face (6 per face) for BW98;
    // the ordered pairs of each bending stencil (12 per stencil) unless bending is off
    const size_t KS = h->d.stretch_model == LCS_STRETCH_SPRING ? 2 * (size_t)h->E : 0;
    const size_t KF = h->d.stretch_model == LCS_STRETCH_BW98 ? 6 * (size_t)h->Fs : 0;
    const size_t KB = h->d.bending_model != LCS_BENDING_NONE ? 12 * (size_t)h->B : 0;
    const size_t KA = 12 * (size_t)h->NB;  // the 12 off-diagonal blocks among each body's DOF slots
    const size_t K = KS + KF + KB + KA;
    auto key_rc = [&](size_t k, uint32_t& r, uint32_t& c) {
        if (k < KS) {
            const uint32_t* e = d->edges + 2 * (k >> 1);
            r = e[k & 1];
            c = e[(k & 1) ^ 1];
        } else if (k < KS + KF) {
            const size_t q = k - KS, f = q / 6, m = q % 6, i = m / 2, jj = m % 2, j = jj < i ? jj : jj + 1;
            r = d->stretch_faces[4 * f + i];
            c = d->stretch_faces[4 * f + j];
        } else if (k < KS + KF + KB) {
            const size_t q = k - KS - KF, st = q / 12, m = q % 12, i = m / 3, jj = m % 3, j = jj < i ? jj : jj + 1;
            r = d->bending[4 * st + i];
            c = d->bending[4 * st + j];
        } else {
            const size_t q = k - KS - KF - KB, bi = q / 12, m = q % 12, i = m / 3, jj = m % 3, j = jj < i ? jj : jj + 1;
            r = d->body_dof[bi] + (uint32_t)i;
            c = d->body_dof[bi] + (uint32_t)j;
        }
    };
    // bucket the columns by row (counting sort), then sort and de-duplicate each row
    std::vector<uint32_t> start(h->V + 1, 0);
    for (size_t k = 0; k < K; ++k) {
        uint32_t r, c;
        key_rc(k, r, c);
        start[r + 1]++;
    }
    for (uint32_t r = 0; r < h->V; ++r) start[r + 1] += start[r];
    std::vector<uint32_t> bucket(K ? K : 1), cursor(start.begin(), start.end() - 1);
    for (size_t k = 0; k < K; ++k) {
        uint32_t r, c;
        key_rc(k, r, c);
        bucket[cursor[r]++] = c;
    }
    std::vector<uint32_t> ucount(h->V, 0);
    parallel_ranges(h->V, [&](size_t rb, size_t re) {
        for (size_t r = rb; r < re; ++r) {
            uint32_t* b0 = bucket.data() + start[r];
            uint32_t* b1 = bucket.data() + start[r + 1];
            std::sort(b0, b1);
            ucount[r] = (uint32_t)(std::unique(b0, b1) - b0);
        }
    });
    std::vector<uint32_t> rp(h->V + 1, 0);
    for (uint32_t r = 0; r < h->V; ++r) rp[r + 1] = rp[r] + ucount[r];
    const size_t nnz = rp[h->V];
    h->nnz_mat = (uint32_t)nnz;
    std::vector<uint32_t> col(nnz ? nnz : 1);
    parallel_ranges(h->V, [&](size_t rb, size_t re) {
        for (size_t r = rb; r < re; ++r) std::copy(bucket.begin() + start[r], bucket.begin() + start[r] + ucount[r], col.begin() + rp[r]);
    });
    // CSR slot of contribution k: its column's position in its row (rows hold about a dozen blocks)
    auto slot_of = [&](size_t k) -> uint32_t {
        uint32_t r, c;
        key_rc(k, r, c);
        const uint32_t* b = col.data() + rp[r];
        const uint32_t n = rp[r + 1] - rp[r];
        uint32_t j = 0;
        while (j < n && b[j] != c) ++j;
        return rp[r] + j;
    };
    // block base offset into mat_val for CSR block j: CSR 9 j (components contiguous) or, in the
    // SELL-32 layout with 4-slot groups, ((g * 9) * 32 + lane) * 4 + slot % 4 for group g = slot / 4
    // (components 128 floats apart; the row-resident PCG reads a group with float4 loads)
    std::vector<uint32_t> base(nnz ? nnz : 1);
    std::vector<uint32_t> sell_ptr, sell_col;
    if (h->sell) {
        const uint32_t ns = (h->V + 31) / 32;
        sell_ptr.assign(ns + 1, 0);
        for (uint32_t s = 0; s < ns; ++s) {
            uint32_t w = 0;
            for (uint32_t r = 32 * s; r < std::min(h->V, 32 * s + 32); ++r) w = std::max(w, rp[r + 1] - rp[r]);
            sell_ptr[s + 1] = sell_ptr[s] + ((w + 3u) & ~3u);
        }
        sell_col.assign(32 * (size_t)sell_ptr[ns], 0);
        for (uint32_t s = 0; s < ns; ++s)
            for (uint32_t lane = 0; lane < 32; ++lane) {
                const uint32_t r = 32 * s + lane;
                const uint32_t len = r < h->V ? rp[r + 1] - rp[r] : 0;
                const uint32_t pad = r < h->V ? r : h->V - 1;  // zero block against a valid row
                for (uint32_t k = 0; k < sell_ptr[s + 1] - sell_ptr[s]; ++k) {
                    const size_t slot = (size_t)sell_ptr[s] + k, g = slot / 4, j = slot % 4;
                    sell_col[(g * 32 + lane) * 4 + j] = k < len ? col[rp[r] + k] : pad;
                    if (k < len) base[rp[r] + k] = (uint32_t)((g * 9 * 32 + lane) * 4 + j);
                }
            }
        h->sell_vals = 9ull * 32 * sell_ptr[ns];
    } else {
        for (size_t j = 0; j < nnz; ++j) base[j] = (uint32_t)(9 * j);
        h->sell_vals = 9ull * nnz;
    }
    std::vector<uint32_t> ss(KS ? KS : 1), fs(KF ? KF : 1), bs(KB ? KB : 1), as(KA ? KA : 1);
    parallel_ranges(K, [&](size_t kb, size_t ke) {
        for (size_t k = kb; k < ke; ++k) {
            const uint32_t v = base[slot_of(k)];
            if (k < KS) ss[k] = v;
            else if (k < KS + KF) fs[k - KS] = v;
            else if (k < KS + KF + KB) bs[k - KS - KF] = v;
            else as[k - KS - KF - KB] = v;
        }
    });
    if (h->det) {
        // per material block (CSR position j): its contributions in contribution order -- springs, faces,
        // stencils, each by element and then by local pair -- the order the gather sums them in
        const size_t KE = KS + KF + KB;
        std::vector<uint32_t> jof(KE ? KE : 1);
        parallel_ranges(KE, [&](size_t kb, size_t ke) {
            for (size_t k = kb; k < ke; ++k) jof[k] = slot_of(k);
        });
        std::vector<uint32_t> bptr(nnz + 1, 0);
        for (size_t k = 0; k < KE; ++k) bptr[jof[k] + 1]++;
        for (size_t j = 0; j < nnz; ++j) bptr[j + 1] += bptr[j];
        std::vector<uint2> bent(KE ? KE : 1);
        std::vector<uint32_t> cur(bptr.begin(), bptr.end() - 1);
        const uint32_t bkind = h->d.bending_model == LCS_BENDING_QUADRATIC ? 3u : 2u;
        for (size_t k = 0; k < KE; ++k) {
            uint2 en;
            if (k < KS) en = make_uint2((uint32_t)(k >> 1), 0u << 4 | (uint32_t)(k & 1));
            else if (k < KS + KF) en = make_uint2((uint32_t)((k - KS) / 6), 1u << 4 | (uint32_t)((k - KS) % 6));
            else en = make_uint2((uint32_t)((k - KS - KF) / 12), bkind << 4 | (uint32_t)((k - KS - KF) % 12));
            bent[cur[jof[k]]++] = en;
        }
        // per vertex: its springs (end 0 or 1), faces (corner 0..2) and stencils (vertex 0..3), in that order
        std::vector<uint32_t> vptr(h->V + 1, 0);
        auto each_vertex_entry = [&](auto&& f) {
            if (KS)
                for (uint32_t e = 0; e < h->E; ++e)
                    for (uint32_t a = 0; a < 2; ++a) f(d->edges[2 * e + a], make_uint2(e, 0u << 4 | a));
            if (KF)
                for (uint32_t fc = 0; fc < h->Fs; ++fc)
                    for (uint32_t a = 0; a < 3; ++a) f(d->stretch_faces[4 * fc + a], make_uint2(fc, 1u << 4 | a));
            if (KB)
                for (uint32_t st = 0; st < h->B; ++st)
                    for (uint32_t a = 0; a < 4; ++a) f(d->bending[4 * st + a], make_uint2(st, bkind << 4 | a));
        };
        each_vertex_entry([&](uint32_t v, uint2) { vptr[v + 1]++; });
        for (uint32_t v = 0; v < h->V; ++v) vptr[v + 1] += vptr[v];
        std::vector<uint2> vent(vptr[h->V] ? vptr[h->V] : 1);
        std::vector<uint32_t> vc(vptr.begin(), vptr.end() - 1);
        each_vertex_entry([&](uint32_t v, uint2 en) { vent[vc[v]++] = en; });
        h->det_nblk = (uint32_t)nnz;
        h->det_off_face = KS ? 12 * (size_t)h->E : 0;
        h->det_off_bend = h->det_off_face + (KF ? 64 * (size_t)h->Fs : 0);
        const size_t nel = h->det_off_bend + (KB ? 16 * (size_t)h->B : 0);
        if (upload(h->det_bptr, bptr.data(), bptr.size()) != cudaSuccess ||
            upload(h->det_bent, bent.data(), bent.size()) != cudaSuccess ||
            upload(h->det_bbase, base.data(), base.size()) != cudaSuccess ||
            upload(h->det_vptr, vptr.data(), vptr.size()) != cudaSuccess ||
            upload(h->det_vent, vent.data(), vent.size()) != cudaSuccess || dalloc(h->det_el, nel ? nel : 1) != cudaSuccess)
            return lcs_fail(LCS_ERR_CUDA, "lcs_newton: deterministic assembly tables: upload failed");
    }
    if (upload(h->mat_rp, rp.data(), rp.size()) != cudaSuccess || upload(h->mat_col, col.data(), col.size()) != cudaSuccess ||
        upload(h->spring_slots, ss.data(), ss.size()) != cudaSuccess ||
        upload(h->face_slots, fs.data(), fs.size()) != cudaSuccess ||
        upload(h->bend_slots, bs.data(), bs.size()) != cudaSuccess ||
        upload(h->body_slots, as.data(), as.size()) != cudaSuccess || dalloc(h->mat_val, h->sell_vals) != cudaSuccess)
        return lcs_fail(LCS_ERR_CUDA, "lcs_newton: material pattern upload failed");
    if (h->sell && (upload(h->sell_ptr, sell_ptr.data(), sell_ptr.size()) != cudaSuccess ||
                    upload(h->sell_col, sell_col.data(), sell_col.size()) != cudaSuccess))
        return lcs_fail(LCS_ERR_CUDA, "lcs_newton: SELL pattern upload failed");
    return LCS_OK;
}

inline int grid256(uint64_t n) { return grid_for(n, 256); }

void mark(lcs_newton* h, int phase)
{
    if (h->profile) cudaEventRecord(h->ev[phase], h->s);
}

// LCS_NEWTON_DETERMINISTIC: the contact pairs into canonical order (two stable radix passes over 42 + 44 key
// bits, then a gather into the scratch list, which becomes the pair list)
int det_sort_pairs(lcs_newton* h)
{
    cudaStream_t s = h->s;
    const uint32_t cap = h->cap_pairs;
    const uint32_t* cnt = &h->st->cnt[2];
    k_pair_keys<<<grid256(cap), 256, 0, s>>>(h->pairs, cnt, cap, 0, nullptr, h->det_keys, h->det_vals, h->det_n);
    lcs_count_launch();
    const bool alt = rs::sort_pairs<uint64_t>(h->det_keys, h->det_vals, h->det_keys_alt, h->det_vals_alt, h->det_n, 0,
                                              cap, 0, 42, h->det_hist, s);
    const uint32_t* ord = alt ? h->det_vals_alt : h->det_vals;
    uint64_t* k2 = alt ? h->det_keys : h->det_keys_alt;
    uint32_t* v2 = alt ? h->det_vals : h->det_vals_alt;
    uint64_t* k3 = alt ? h->det_keys_alt : h->det_keys;
    uint32_t* v3 = alt ? h->det_vals_alt : h->det_vals;
    k_pair_keys<<<grid256(cap), 256, 0, s>>>(h->pairs, cnt, cap, 1, ord, k2, v2, h->det_n);
    lcs_count_launch();
    const bool alt2 = rs::sort_pairs<uint64_t>(k2, v2, k3, v3, h->det_n, 0, cap, 0, 44, h->det_hist, s);
    k_pair_gather<<<grid256(cap), 256, 0, s>>>(h->pairs, h->det_n, alt2 ? v3 : v2, h->det_pairs);
    lcs_count_launch();
    std::swap(h->pairs, h->det_pairs);
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

// LCS_NEWTON_DETERMINISTIC: the contact gradient and diagonal blocks, summed per row in canonical pair order
int det_contact_rows(lcs_newton* h, cudaStream_t s)
{
    const uint32_t cap4 = 4 * h->cap_pairs;
    k_cg_keys<<<grid256(h->cap_pairs), 256, 0, s>>>(h->pairs, h->det_n, h->V, h->det_keys, h->det_vals, h->det_n + 1);
    lcs_count_launch();
    int bits = 1;
    while (bits < 40 && (1ull << bits) <= h->V) ++bits;
    const bool alt = rs::sort_pairs<uint64_t>(h->det_keys, h->det_vals, h->det_keys_alt, h->det_vals_alt, h->det_n + 1,
                                              0, cap4, 0, bits, h->det_hist, s);
    k_cg_rows<<<grid256(cap4), 256, 0, s>>>(alt ? h->det_keys_alt : h->det_keys, alt ? h->det_vals_alt : h->det_vals,
                                            h->det_n + 1, h->V, h->pairs, h->b, h->diag);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

// counts the plain comparator reads back where the reference does (download_*_count)
int host_readback(lcs_newton* h)
{
    LCS_CUDA_TRY(cudaMemcpyAsync(h->h_st, h->st, sizeof(Status), cudaMemcpyDeviceToHost, h->s));
    if (h->batch) {
        LCS_CUDA_TRY(cudaMemcpyAsync(h->h_bsc, h->bsc, 3 * sizeof(float) * h->S, cudaMemcpyDeviceToHost, h->s));
        LCS_CUDA_TRY(cudaMemcpyAsync(h->h_bpcg, h->bpcg, sizeof(lcs_pcg_stats) * h->S, cudaMemcpyDeviceToHost, h->s));
    }
    LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    return LCS_OK;
}

// the plain loop's host copies of a position-sized vector (pinned mirror)
int copy_x_to_host(lcs_newton* h, const float4* src)
{
    LCS_CUDA_TRY(cudaMemcpyAsync(h->h_x_iter, src, 16 * (size_t)h->V, cudaMemcpyDeviceToHost, h->s));
    LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    return LCS_OK;
}

// refit + queries of both trees; lists into out_vf / out_ee; *capped |= 1 when a traversal ended early
// EE candidates of the edge tree (fused mode: the once-per-pair traversal where it applies)
int query_ee(lcs_newton* h, const float* X0, const float* X1, const uint32_t* ED, uint32_t* PE, uint32_t* cnt_ee,
             uint32_t* capped, cudaStream_t s)
{
    if (h->ee_sym && !h->plain && !h->full_traversal)
        return lcs_bvh_query_ee_sym_capped(h->edge_tree, X0, X1, ED, h->ee_dhat, PE, h->cap_ee, cnt_ee, capped, s);
    return lcs_bvh_query_ee_capped(h->edge_tree, X0, X1, ED, h->E, h->dhat, h->offset, PE, h->cap_ee, cnt_ee, capped, s);
}

int broad_phase(lcs_newton* h, const float4* x0, const float4* x1, uint2* out_vf, uint2* out_ee, uint32_t* cnt_vf,
                uint32_t* cnt_ee, uint32_t* capped)
{
    const float* X0 = reinterpret_cast<const float*>(x0);
    const float* X1 = reinterpret_cast<const float*>(x1);
    uint32_t* PV = reinterpret_cast<uint32_t*>(out_vf);
    uint32_t* PE = reinterpret_cast<uint32_t*>(out_ee);
    const uint32_t* FA = reinterpret_cast<const uint32_t*>(h->faces);
    const uint32_t* ED = reinterpret_cast<const uint32_t*>(h->edges);
    int rc;
    if (h->batch) {  // forests of per-scene trees, same two lanes
        LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
        LCS_CUDA_TRY(cudaStreamWaitEvent(h->s2, h->fork, 0));
        if ((rc = lcs_forest_update_refit(h->edge_forest, h->offset, X0, X1, ED, h->s2))) return rc;
        if ((rc = lcs_forest_query_ee_capped(h->edge_forest, X0, X1, ED, h->dhat, h->offset, PE, h->cap_ee, cnt_ee,
                                             capped, h->s2)))
            return rc;
        if ((rc = lcs_forest_update_refit(h->face_forest, h->offset, X0, X1, FA, h->s))) return rc;
        if ((rc = lcs_forest_query_vf_capped(h->face_forest, X0, X1, h->V, h->vscene, h->dhat, h->offset, PV, h->cap_vf,
                                             cnt_vf, capped, h->s)))
            return rc;
        LCS_CUDA_TRY(cudaEventRecord(h->join, h->s2));
        LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
        return LCS_OK;
    }
    if (!h->plain && h->s2) {
        // two independent lanes: face tree + VF queries here, edge tree + EE queries on s2; both are
        // latency-bound tree walks that leave most of the GPU idle when run one after the other
        LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
        LCS_CUDA_TRY(cudaStreamWaitEvent(h->s2, h->fork, 0));
        if ((rc = lcs_bvh_update_refit(h->edge_tree, h->offset, X0, X1, ED, h->s2))) return rc;
        if ((rc = query_ee(h, X0, X1, ED, PE, cnt_ee, capped, h->s2))) return rc;
        if ((rc = lcs_bvh_update_refit(h->face_tree, h->offset, X0, X1, FA, h->s))) return rc;
        if ((rc = lcs_bvh_query_vf_capped(h->face_tree, X0, X1, h->V, h->dhat, h->offset, PV, h->cap_vf, cnt_vf, capped,
                                          h->s)))
            return rc;
        LCS_CUDA_TRY(cudaEventRecord(h->join, h->s2));
        LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
        return LCS_OK;
    }
    if (h->plain) {
        if ((rc = lcs_bvh_update_leaves(h->face_tree, h->offset, X0, X1, FA, h->s))) return rc;
        if ((rc = lcs_bvh_refit(h->face_tree, h->s))) return rc;
    } else if ((rc = lcs_bvh_update_refit(h->face_tree, h->offset, X0, X1, FA, h->s))) {
        return rc;
    }
    if ((rc = lcs_bvh_query_vf_capped(h->face_tree, X0, X1, h->V, h->dhat, h->offset, PV, h->cap_vf, cnt_vf, capped, h->s)))
        return rc;
    if (h->plain) {
        if ((rc = lcs_bvh_update_leaves(h->edge_tree, h->offset, X0, X1, ED, h->s))) return rc;
        if ((rc = lcs_bvh_refit(h->edge_tree, h->s))) return rc;
    } else if ((rc = lcs_bvh_update_refit(h->edge_tree, h->offset, X0, X1, ED, h->s))) {
        return rc;
    }
    return query_ee(h, X0, X1, ED, PE, cnt_ee, capped, h->s);
}

// DCD candidates of iterate x from the previous iteration's CCD lists (swept from x_iter to x_iter + dx,
// so they contain every static-box overlap at x = x_iter + toi dx, 0 <= toi <= 1), in the two lanes
int dcd_by_filter(lcs_newton* h)
{
    const float* X = reinterpret_cast<const float*>(h->x);
    int rc;
    LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
    LCS_CUDA_TRY(cudaStreamWaitEvent(h->s2, h->fork, 0));
    if ((rc = lcs_candidates_filter(1, reinterpret_cast<const uint32_t*>(h->bp_ee), h->prev_ccd + 1, h->cap_ee, X,
                                    reinterpret_cast<const uint32_t*>(h->edges), h->dhat, h->offset,
                                    reinterpret_cast<uint32_t*>(h->dcd_ee), h->cap_ee, &h->st->cnt[1], h->s2)))
        return rc;
    if ((rc = lcs_candidates_filter(0, reinterpret_cast<const uint32_t*>(h->bp_vf), h->prev_ccd, h->cap_vf, X,
                                    reinterpret_cast<const uint32_t*>(h->faces), h->dhat, h->offset,
                                    reinterpret_cast<uint32_t*>(h->dcd_vf), h->cap_vf, &h->st->cnt[0], h->s)))
        return rc;
    LCS_CUDA_TRY(cudaEventRecord(h->join, h->s2));
    LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
    return LCS_OK;
}

// A batch with affine bodies: its scenes without bodies filter the previous CCD lists (exact, as above),
// its scenes with bodies -- whose rigid vertices are placed by p + A x_bar and may round outside the swept
// boxes -- are traversed again with static boxes; both append to the same DCD lists.
int dcd_mixed(lcs_newton* h)
{
    const float* X = reinterpret_cast<const float*>(h->x);
    const uint32_t* ED = reinterpret_cast<const uint32_t*>(h->edges);
    const uint32_t* FA = reinterpret_cast<const uint32_t*>(h->faces);
    int rc;
    LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
    LCS_CUDA_TRY(cudaStreamWaitEvent(h->s2, h->fork, 0));
    if ((rc = lcs_candidates_filter_masked(1, reinterpret_cast<const uint32_t*>(h->bp_ee), h->prev_ccd + 1, h->cap_ee, X,
                                           ED, h->dhat, h->offset, reinterpret_cast<uint32_t*>(h->dcd_ee), h->cap_ee,
                                           &h->st->cnt[1], h->s2, h->rigid_scene_v)))
        return rc;
    if ((rc = lcs_forest_update_refit(h->edge_forest, h->offset, X, X, ED, h->s2))) return rc;
    if ((rc = lcs_forest_query_ee_capped(h->edge_forest, X, X, ED, h->dhat, h->offset,
                                         reinterpret_cast<uint32_t*>(h->dcd_ee), h->cap_ee, &h->st->cnt[1], nullptr,
                                         h->s2, h->rigid_scene_v)))
        return rc;
    if ((rc = lcs_candidates_filter_masked(0, reinterpret_cast<const uint32_t*>(h->bp_vf), h->prev_ccd, h->cap_vf, X, FA,
                                           h->dhat, h->offset, reinterpret_cast<uint32_t*>(h->dcd_vf), h->cap_vf,
                                           &h->st->cnt[0], h->s, h->rigid_scene_v)))
        return rc;
    if ((rc = lcs_forest_update_refit(h->face_forest, h->offset, X, X, FA, h->s))) return rc;
    if ((rc = lcs_forest_query_vf_capped(h->face_forest, X, X, h->V, h->vscene, h->dhat, h->offset,
                                         reinterpret_cast<uint32_t*>(h->dcd_vf), h->cap_vf, &h->st->cnt[0], nullptr,
                                         h->s, h->rigid_scene_v)))
        return rc;
    LCS_CUDA_TRY(cudaEventRecord(h->join, h->s2));
    LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
    return LCS_OK;
}

bool grow(lcs_newton* h)
{
    const Status& s = *h->h_st;
    bool g = false;
    const uint32_t need_vf = std::max(s.cnt[0], s.cnt[3]), need_ee = std::max(s.cnt[1], s.cnt[4]);
    while (need_vf > h->cap_vf) { h->cap_vf *= 2; g = true; }
    while (need_ee > h->cap_ee) { h->cap_ee *= 2; g = true; }
    while (s.cnt[2] > h->cap_pairs) { h->cap_pairs *= 2; g = true; }
    return g;
}

LsArgs ls_args(const lcs_newton* h)
{
    const lcs_scene_desc& d = h->d;
    LsArgs a{};
    a.V = h->V;
    a.x0 = h->x_iter;
    a.dx = h->dx;
    a.xt = h->x_tilde;
    a.rest = h->rest;
    a.mass = h->mass;
    a.pinned = h->pinned;
    a.h2inv = 1.0f / (d.dt * d.dt);
    a.dirichlet = d.dirichlet;
    if (d.stretch_model == LCS_STRETCH_SPRING) {
        a.E = h->E;
        a.edges = h->edges;
        a.rest_len = h->rest_len;
        a.spring_k = d.spring_k;
        a.spring_kper = h->spring_kper;
    } else {
        a.ml = h->ml;
        a.Fs = h->Fs;
        a.sfaces = h->sfaces;
        a.dm = h->dm;
        a.sarea = h->sarea;
        a.mu = d.stretch_mu;
        a.lambda = d.stretch_lambda;
    }
    if (d.bending_model != LCS_BENDING_NONE) {
        a.B = h->B;
        a.bend = h->bend;
        a.rest_angle = h->rest_angle;
        a.hbar = h->hbar;
        a.Q = h->Q;
        a.kb = d.bending_k;
        a.bend_kper = h->bend_kper;
        a.bend_scaling = d.bending_scaling;
        a.bending_model = d.bending_model;
    }
    a.P = h->cap_pairs;
    a.pairs = h->pairs;
    a.pair_count = &h->st->cnt[2];
    a.dhat = h->dhat;
    a.offset = h->offset;
    a.abd = abd_of(h);
    a.NB = h->NB;
    a.bmass = h->bmass;
    a.bvol = h->bvol;
    a.bkappa = h->bkappa;
    return a;
}

int ls_grid(const lcs_newton* h)
{
    const uint32_t n = std::max(std::max(std::max(h->V, h->Fs), std::max(h->E, h->B)), std::max(h->cap_pairs, h->NB));
    return grid_for(n, 256, 4);
}

// one round of the fused energy line search on the device: E at alpha = 0 and kLsSlots - 1 halvings
// starting at toi / 2^j0, then the pick (st->alpha, st->ls_state)
int ls_round(lcs_newton* h, int j0)
{
    LCS_CUDA_TRY(cudaMemsetAsync(h->ls_E, 0, sizeof(double) * kLsSlots, h->s));
    k_ls_energy<kLsSlots><<<ls_grid(h), 256, 0, h->s>>>(ls_args(h), j0, h->st, h->ls_E);
    lcs_count_launch();
    k_ls_pick<<<1, 1, 0, h->s>>>(h->ls_E, j0, 1e-2f * h->d.dt, h->st);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

// the reference's sequence for the plain loop: one step length per energy evaluation, each read
// back to the host (newton_solver.cpp:3790-3834); toi and max |dx| are on the host already
int plain_line_search(lcs_newton* h)
{
    const Status& s = *h->h_st;
    float alpha = s.toi;
    int j = 0;
    if (!(s.max_dx < 1e-2f * h->d.dt)) {
        const LsArgs a = ls_args(h);
        for (int count = 0; count < 20; ++count) {
            LCS_CUDA_TRY(cudaMemsetAsync(h->ls_E, 0, sizeof(double) * 2, h->s));
            k_ls_energy<2><<<ls_grid(h), 256, 0, h->s>>>(a, j, h->st, h->ls_E);
            lcs_count_launch();
            LCS_LAUNCH_CHECK();
            LCS_CUDA_TRY(cudaMemcpyAsync(h->h_ls_E, h->ls_E, sizeof(double) * 2, cudaMemcpyDeviceToHost, h->s));
            LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
            if (h->h_ls_E[1] < h->h_ls_E[0] + (double)1.19209290E-7f) break;
            alpha /= 2.0f;
            ++j;
            if (alpha < 1e-4f) return lcs_fail(LCS_ERR_LINESEARCH, "lcs_newton: energy line search failed (step below 1e-4)");
        }
    }
    *h->h_alpha = alpha;
    LCS_CUDA_TRY(cudaMemcpyAsync(&h->st->alpha, h->h_alpha, sizeof(float), cudaMemcpyHostToDevice, h->s));
    h->ls_halvings += j;
    return LCS_OK;
}

// one Newton iteration (the body of the loop in physics_step_GPU); returns LCS_OK or an error
int newton_iteration(lcs_newton* h)
{
    const uint32_t V = h->V;
    const lcs_scene_desc& d = h->d;
    int rc;
    for (int attempt = 0; attempt < 8; ++attempt) {
        if (attempt) {
            h->retries++;
            h->filter_ok = false;  // the CCD lists of the undone iteration do not describe this iterate
        }
        const bool filter = !h->plain && !h->full_traversal && h->filter_ok;
        if (filter) {
            k_save_ccd_counts<<<1, 1, 0, h->s>>>(h->st, h->prev_ccd);
            lcs_count_launch();
        }
        mark(h, kPhMaterial);
        k_reset_status<<<1, 32, 0, h->s>>>(h->st);
        lcs_count_launch();
        if (h->batch) {
            k_b_reset<<<grid_for(h->S, 256), 256, 0, h->s>>>(h->S, h->bsc);
            lcs_count_launch();
        }
        if (h->plain) {  // x_iter_start copied to the host for host_apply_dx (newton_solver.cpp:4196-4198)
            if ((rc = copy_x_to_host(h, h->x))) return rc;
        }
        // the material producers (inertia, elastic energies, bodies) touch b, the diagonal and the material
        // blocks only: beside the DCD broad and narrow phases on s3 (fused mode), joined before assembly
        cudaStream_t ms = h->s3 ? h->s3 : h->s;
        if (ms != h->s) {
            LCS_CUDA_TRY(cudaEventRecord(h->fork_m, h->s));
            LCS_CUDA_TRY(cudaStreamWaitEvent(ms, h->fork_m, 0));
        }
        k_inertia<<<grid256(V), 256, 0, ms>>>(V, d.dt, d.dirichlet, h->mass, h->pinned, h->x, h->x_tilde, h->x_iter, h->b,
                                          h->diag, d.use_floor, d.floor_y, d.kappa, h->vert_area, h->dhat, h->offset, abd_of(h));
        lcs_count_launch();
        LCS_CUDA_TRY(cudaMemsetAsync(h->mat_val, 0, sizeof(float) * h->sell_vals, ms));
        const uint32_t cs = h->sell ? 128u : 1u;
        if (h->det) {  // per-element terms, then per-row and per-block sums in element order
            if (h->E && d.stretch_model == LCS_STRETCH_SPRING) {
                k_springs_det<<<grid256(h->E), 256, 0, ms>>>(h->E, h->edges, h->rest_len, h->spring_kper, d.spring_k,
                                                               h->x, h->det_el);
                lcs_count_launch();
            }
            if (h->Fs && d.stretch_model == LCS_STRETCH_BW98) {
                k_stretch_bw98_det<<<grid256(h->Fs), 256, 0, ms>>>(h->Fs, h->sfaces, h->dm, h->sarea, h->ml, d.stretch_mu,
                                                                     d.stretch_lambda, h->x, h->det_el + h->det_off_face);
                lcs_count_launch();
            }
            if (h->B && d.bending_model == LCS_BENDING_DIHEDRAL) {
                k_bending_dihedral_det<<<grid256(h->B), 256, 0, ms>>>(h->B, h->bend, h->rest_angle, h->hbar, h->bend_kper,
                                                                        d.bending_k, d.bending_scaling, h->x,
                                                                        h->det_el + h->det_off_bend);
                lcs_count_launch();
            } else if (h->B && d.bending_model == LCS_BENDING_QUADRATIC) {
                k_bending_det<<<grid256(h->B), 256, 0, ms>>>(h->B, h->bend, h->Q, d.bending_k, h->x, h->rest,
                                                             h->det_el + h->det_off_bend);
                lcs_count_launch();
            }
            const DetEl D{h->det_el, h->det_off_face, h->det_off_bend, h->Q, d.bending_k};
            k_det_rows<<<grid256(V), 256, 0, ms>>>(V, h->det_vptr, h->det_vent, D, h->b, h->diag);
            lcs_count_launch();
            if (h->det_nblk) {
                k_det_blocks<<<grid256(h->det_nblk), 256, 0, ms>>>(h->det_nblk, h->det_bptr, h->det_bent, h->det_bbase, D,
                                                                     cs, h->mat_val);
                lcs_count_launch();
            }
        }
        if (!h->det && h->E && d.stretch_model == LCS_STRETCH_SPRING) {
            k_springs<<<grid256(h->E), 256, 0, ms>>>(h->E, h->edges, h->rest_len, h->spring_kper, d.spring_k, h->x,
                                                       h->b, h->diag, h->spring_slots, cs, h->mat_val);
            lcs_count_launch();
        }
        if (!h->det && h->Fs && d.stretch_model == LCS_STRETCH_BW98) {
            k_stretch_bw98<<<grid256(h->Fs), 256, 0, ms>>>(h->Fs, h->sfaces, h->dm, h->sarea, h->ml, d.stretch_mu,
                                                             d.stretch_lambda, h->x, h->b, h->diag, h->face_slots, cs,
                                                             h->mat_val);
            lcs_count_launch();
        }
        if (h->det) {
        } else if (h->B && d.bending_model == LCS_BENDING_DIHEDRAL) {
            k_bending_dihedral<<<grid256(h->B), 256, 0, ms>>>(h->B, h->bend, h->rest_angle, h->hbar, h->bend_kper,
                                                                d.bending_k, d.bending_scaling, h->x, h->b, h->diag,
                                                                h->bend_slots, cs, h->mat_val);
            lcs_count_launch();
        } else if (h->B && d.bending_model == LCS_BENDING_QUADRATIC) {
            k_bending<<<grid256(h->B), 256, 0, ms>>>(h->B, h->bend, h->Q, d.bending_k, h->x, h->rest, h->b, h->diag,
                                                 h->bend_slots, cs, h->mat_val);
            lcs_count_launch();
        }
        if (h->NB) {
            k_abd_body<<<grid256(h->NB), 256, 0, ms>>>(h->NB, h->body_dof, h->bmass, h->bvol, h->bkappa, h->bfixed,
                                                         1.0f / (d.dt * d.dt), d.dirichlet, h->x, h->x_tilde, h->b,
                                                         h->diag, h->body_slots, cs, h->mat_val);
            lcs_count_launch();
            if (d.use_floor) {
                k_abd_floor<<<grid256(V), 256, 0, ms>>>(V, abd_of(h), h->pinned, h->x, d.floor_y, d.kappa,
                                                          h->vert_area, h->dhat, h->offset, h->b, h->diag,
                                                          h->body_slots, cs, h->mat_val);
                lcs_count_launch();
            }
        }
        // update_contact_set (newton_solver.cpp:4093-4104)
        mark(h, kPhDcdBroad);
        uint2* dvf = h->plain ? h->bp_vf : h->dcd_vf;
        uint2* dee = h->plain ? h->bp_ee : h->dcd_ee;
        // a single scene filters inside the DCD kernels (no candidate list in between)
        const bool fused_dcd = filter && !h->batch;
        if (fused_dcd) {
            // lcs_dcd_*_filtered below read the previous CCD lists directly
        } else if (filter) {
            if ((rc = h->rigid_scene_v ? dcd_mixed(h) : dcd_by_filter(h))) return rc;
        } else if ((rc = broad_phase(h, h->x, h->x, dvf, dee, &h->st->cnt[0], &h->st->cnt[1], nullptr))) {
            return rc;
        }
        if (h->plain) {
            if ((rc = host_readback(h))) return rc;  // download_broadphase_collision_count
            if (grow(h)) { if ((rc = alloc_contact(h))) return rc; continue; }
        }
        mark(h, kPhDcdNarrow);
        const float* X = reinterpret_cast<const float*>(h->x);
        // fused: the EE pairs on s2 beside the VF pairs (both append through the pair counter)
        const bool dlanes = !h->plain && h->s2;
        if (dlanes) {
            LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
            LCS_CUDA_TRY(cudaStreamWaitEvent(h->s2, h->fork, 0));
        }
        auto dcd_ee = [&](cudaStream_t st) {
            if (fused_dcd)
                return lcs_dcd_ee_filtered(reinterpret_cast<const uint32_t*>(h->bp_ee), h->prev_ccd + 1, h->cap_ee, X,
                                           reinterpret_cast<const uint32_t*>(h->edges), h->body, h->edge_area, h->dhat,
                                           h->offset, d.kappa, h->pairs, h->cap_pairs, &h->st->cnt[2],
                                           &h->st->cnt[1], st);
            return lcs_dcd_ee(reinterpret_cast<uint32_t*>(dee), &h->st->cnt[1], h->cap_ee, X,
                              reinterpret_cast<const uint32_t*>(h->edges), h->body, h->edge_area, h->dhat, h->offset,
                              d.kappa, h->pairs, h->cap_pairs, &h->st->cnt[2], st);
        };
        if (dlanes && (rc = dcd_ee(h->s2))) return rc;
        if (fused_dcd)
            rc = lcs_dcd_vf_filtered(reinterpret_cast<const uint32_t*>(h->bp_vf), h->prev_ccd, h->cap_vf, X,
                                     reinterpret_cast<const uint32_t*>(h->faces), h->body, h->vert_area, h->face_area,
                                     h->dhat, h->offset, d.kappa, h->pairs, h->cap_pairs, &h->st->cnt[2],
                                     &h->st->cnt[0], h->s);
        else
            rc = lcs_dcd_vf(reinterpret_cast<uint32_t*>(dvf), &h->st->cnt[0], h->cap_vf, X,
                            reinterpret_cast<const uint32_t*>(h->faces), h->body, h->vert_area, h->face_area, h->dhat,
                            h->offset, d.kappa, h->pairs, h->cap_pairs, &h->st->cnt[2], h->s);
        if (rc) return rc;
        if (!dlanes && (rc = dcd_ee(h->s))) return rc;  // the reference's order: VF pairs, then EE pairs
        if (dlanes) {
            LCS_CUDA_TRY(cudaEventRecord(h->join, h->s2));
            LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
        }
        if (h->plain) {
            if ((rc = host_readback(h))) return rc;  // download_narrowphase_collision_count
            if (grow(h)) { if ((rc = alloc_contact(h))) return rc; continue; }
        }
        if (h->det && (rc = det_sort_pairs(h))) return rc;
        if (ms != h->s) {
            LCS_CUDA_TRY(cudaEventRecord(h->join_m, ms));
            LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join_m, 0));
        }
        // evaluate_contact (newton_solver.cpp:4105-4120)
        mark(h, kPhAssembly);
        // fused: gradient and diagonal on s2 beside the off-diagonal assembly (disjoint outputs)
        cudaStream_t gs = dlanes ? h->s2 : h->s;
        if (dlanes) {
            LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
            LCS_CUDA_TRY(cudaStreamWaitEvent(gs, h->fork, 0));
        }
        if (h->NB) {  // pairs with a rigid side go to the body's DOF slots (ABD remap)
            const lcs_abd_view av{h->body, reinterpret_cast<const float*>(h->model_x), h->body_dof};
            if ((rc = lcs_contact_grad_diag_abd(h->pairs, &h->st->cnt[2], h->cap_pairs, reinterpret_cast<float*>(h->b),
                                                reinterpret_cast<float*>(h->diag), &av, gs)))
                return rc;
            if ((rc = lcs_contact_offdiag_bsr_abd(h->asmb, h->pairs, &h->st->cnt[2], h->cap_pairs, &av, h->s))) return rc;
        } else {
            if (h->det) {
                if ((rc = det_contact_rows(h, gs))) return rc;
            } else if ((rc = lcs_contact_grad_diag(h->pairs, &h->st->cnt[2], h->cap_pairs,
                                                   reinterpret_cast<float*>(h->b), reinterpret_cast<float*>(h->diag),
                                                   gs))) {
                return rc;
            }
            if ((rc = lcs_contact_offdiag_bsr(h->asmb, h->pairs, &h->st->cnt[2], h->cap_pairs, h->s))) return rc;
        }
        if (dlanes) {
            LCS_CUDA_TRY(cudaEventRecord(h->join, gs));
            LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
        }
        if (h->plain) {  // prescan + construct adjacency + the two-level triplet sort read back counts 4 times
            for (int k = 0; k < 4; ++k)
                if ((rc = host_readback(h))) return rc;
        }
        // linear solve
        mark(h, kPhPcg);
        lcs_bsr A{h->V, h->mat_rp, h->mat_col, h->mat_val};
        lcs_bsr Bc;
        const uint32_t* d_nnzb = nullptr;
        lcs_assembler_bsr(h->asmb, &Bc, &d_nnzb);
        lcs_pcg_opts o{d.pcg_max_iter, d.pcg_rel_tol, d.pcg_abs_rz_tol, h->plain ? d.pcg_check_every : 1,
                       (h->fp64 ? LCS_PCG_FP64_DOTS : 0) | (h->plain ? LCS_PCG_PLAIN : LCS_PCG_NO_STATS) |
                           (h->cg1 ? LCS_PCG_SINGLE_REDUCTION : 0) |
                           (h->global_matrix ? LCS_PCG_INTERNAL_NO_RESIDENT : 0)};
        lcs_pcg_stats ps;
        if (h->batch)
            rc = lcs_pcg_solve_batch(h->pcg, h->S, h->voff_d, h->h_voff.data(), h->active,
                                     reinterpret_cast<const float*>(h->diag), h->nnz_mat ? &A : nullptr, &Bc,
                                     reinterpret_cast<const float*>(h->b), reinterpret_cast<float*>(h->dx), &o, h->bpcg,
                                     h->cluster, h->s);
        else if (h->sell) {
            // the slice-resident solve multiplies the contact blocks from the CSR itself; the others read them as SELL-32
            const bool resident = h->cg1 && !h->global_matrix && lcs_pcg_resident(h->pcg);
            const bool cs = h->cs_val != nullptr && !resident;
            if (cs && (rc = lcs_contact_to_sell(h->V, &Bc, h->cs_width, h->cs_ptr, h->cs_col, h->cs_val, h->cs_cap,
                                                h->cs_ok, h->s)))
                return rc;
            rc = lcs_pcg_solve_sell(h->pcg, reinterpret_cast<const float*>(h->diag), h->sell_ptr, h->sell_col,
                                    h->mat_val, &Bc, reinterpret_cast<const float*>(h->b),
                                    reinterpret_cast<float*>(h->dx), &o, nullptr, h->s, cs ? h->cs_ptr : nullptr,
                                    h->cs_col, h->cs_val, h->cs_ok);
        }
        else
            rc = lcs_pcg_solve(h->pcg, reinterpret_cast<const float*>(h->diag), h->nnz_mat ? &A : nullptr, &Bc,
                               reinterpret_cast<const float*>(h->b), reinterpret_cast<float*>(h->dx), &o,
                               h->plain ? &ps : nullptr, h->s);
        if (rc != LCS_OK && rc != LCS_ERR_NAN) return rc;
        if (!h->batch) {
            k_pcg_to_status<<<1, 1, 0, h->s>>>(lcs_pcg_device_stats(h->pcg), h->st);
            lcs_count_launch();
        }
        if (h->NB) {
            k_abd_expand<<<grid256(V), 256, 0, h->s>>>(V, abd_of(h), h->dx);
            lcs_count_launch();
        }
        if (h->plain) {  // device_solve copies cgX to the host at its end (precond_cg.cpp:757-758)
            if ((rc = copy_x_to_host(h, h->dx))) return rc;
        }
        // line_search (newton_solver.cpp:3685-3884): CCD step bound
        mark(h, kPhCcdBroad);
        if (h->batch)
            k_b_apply_unit<<<grid256(V), 256, 0, h->s>>>(V, h->vscene, h->S, h->x_iter, h->dx, h->x, h->bsc, abd_of(h));
        else
            k_apply_unit<<<grid256(V), 256, 0, h->s>>>(V, h->x_iter, h->dx, h->x, h->st, abd_of(h));
        lcs_count_launch();
        if ((rc = broad_phase(h, h->x_iter, h->x, h->bp_vf, h->bp_ee, &h->st->cnt[3], &h->st->cnt[4],
                              h->plain ? nullptr : &h->st->cnt[5])))
            return rc;
        if (h->plain) {
            if ((rc = host_readback(h))) return rc;
            if (grow(h)) {
                k_copy4<<<grid256(V), 256, 0, h->s>>>(V, h->x_iter, h->x);
                lcs_count_launch();
                if ((rc = alloc_contact(h))) return rc;
                continue;
            }
        }
        mark(h, kPhCcdNarrow);
        const float* XI = reinterpret_cast<const float*>(h->x_iter);
        const int ccd_flags = h->fp64 ? LCS_CCD_FP64 : 0;
        if (d.use_floor) {
            k_floor_ccd<<<grid256(V), 256, 0, h->s>>>(V, h->x_iter, h->x, h->offset, h->pinned, d.floor_y, h->st);
            lcs_count_launch();
        }
        // fused mode: the EE step bound runs beside the VF one (both only lower the same minimum)
        const bool lanes = !h->plain && h->s2;
        cudaStream_t s_ee = lanes ? h->s2 : h->s;
        if (lanes) {
            LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
            LCS_CUDA_TRY(cudaStreamWaitEvent(h->s2, h->fork, 0));
        }
        if (h->batch) {
            if ((rc = lcs_ccd_batch(1, reinterpret_cast<uint32_t*>(h->bp_ee), &h->st->cnt[4], h->cap_ee, XI, X,
                                    reinterpret_cast<const uint32_t*>(h->edges), h->body, h->offset, h->vscene, h->bsc,
                                    nullptr, ccd_flags, s_ee)))
                return rc;
            if ((rc = lcs_ccd_batch(0, reinterpret_cast<uint32_t*>(h->bp_vf), &h->st->cnt[3], h->cap_vf, XI, X,
                                    reinterpret_cast<const uint32_t*>(h->faces), h->body, h->offset, h->vscene, h->bsc,
                                    nullptr, ccd_flags, h->s)))
                return rc;
        } else {
            if ((rc = lcs_ccd_ee(reinterpret_cast<uint32_t*>(h->bp_ee), &h->st->cnt[4], h->cap_ee, XI, X, reinterpret_cast<const uint32_t*>(h->edges), h->body, h->offset,
                                 &h->st->toi, nullptr, ccd_flags, s_ee)))
                return rc;
            if ((rc = lcs_ccd_vf(reinterpret_cast<uint32_t*>(h->bp_vf), &h->st->cnt[3], h->cap_vf, XI, X, reinterpret_cast<const uint32_t*>(h->faces), h->body, h->offset,
                                 &h->st->toi, nullptr, ccd_flags, h->s)))
                return rc;
        }
        if (lanes) {
            LCS_CUDA_TRY(cudaEventRecord(h->join, h->s2));
            LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
        }
        if (h->plain)
            if ((rc = host_readback(h))) return rc;  // ccd_get_toi
        if (h->energy_ls) {
            if ((rc = h->plain ? plain_line_search(h) : ls_round(h, 0))) return rc;
        }
        mark(h, kPhApply);
        if (h->batch)
            k_b_apply_final<<<grid256(V), 256, 0, h->s>>>(V, h->vscene, h->S, h->x_iter, h->dx, h->x, h->pinned, h->x_tilde,
                                                    h->bsc, abd_of(h));
        else
            k_apply_final<<<grid256(V), 256, 0, h->s>>>(V, h->x_iter, h->dx, h->x, h->pinned, h->x_tilde, h->st,
                                                  h->energy_ls, abd_of(h));
        lcs_count_launch();
        LCS_LAUNCH_CHECK();
        mark(h, kPhases);
        if ((rc = host_readback(h))) return rc;  // the one read-back of the fused loop
        if (h->profile) {
            for (int p = kPhMaterial; p < kPhases; ++p) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, h->ev[p], h->ev[p + 1 < kPhases ? p + 1 : kPhases]);
                h->phase_ms[p] += ms;
                h->phase_launch_count[p] += 1;
            }
        }
        // the next iteration may filter these CCD lists if no traversal ended early
        // (not with affine bodies: their vertices are placed by p + A x_bar of the stepped q, which may round
        // outside the swept box of x_iter + t dx by an ulp)
        // (a batch with bodies filters its other scenes and traverses those, dcd_mixed)
        h->filter_ok = !h->plain && (!h->NB || h->batch) && h->h_st->cnt[5] == 0u;
        if (grow(h)) {  // an overflow anywhere: undo the step and run the iteration again
            k_copy4<<<grid256(V), 256, 0, h->s>>>(V, h->x_iter, h->x);
            lcs_count_launch();
            if ((rc = alloc_contact(h))) return rc;
            continue;
        }
        if (h->batch) {
            for (uint32_t sc = 0; sc < h->S; ++sc)
                if (h->h_bpcg[sc].status == LCS_ERR_NAN) return lcs_fail(LCS_ERR_NAN, "lcs_newton: NaN/Inf in PCG");
        } else if (h->h_st->pcg_status == LCS_ERR_NAN) {
            return lcs_fail(LCS_ERR_NAN, "lcs_newton: NaN/Inf in PCG");
        }
        if (h->energy_ls && !h->plain) {
            // rare: no step length of the first round lowered the energy; continue with the next halvings
            for (int round = 1; h->h_st->ls_state == 2; ++round) {
                if ((rc = ls_round(h, round * (kLsSlots - 1)))) return rc;
                k_apply_final<<<grid256(V), 256, 0, h->s>>>(V, h->x_iter, h->dx, h->x, h->pinned, h->x_tilde, h->st, 1,
                                                            abd_of(h));
                lcs_count_launch();
                if ((rc = host_readback(h))) return rc;
            }
            if (h->h_st->ls_state == 3)
                return lcs_fail(LCS_ERR_LINESEARCH, "lcs_newton: energy line search failed (step below 1e-4)");
            h->ls_halvings += h->h_st->ls_iters;
        }
        h->last_alpha = h->energy_ls ? h->h_st->alpha : h->h_st->toi;
        return LCS_OK;
    }
    return lcs_fail(LCS_ERR_CAPACITY, "lcs_newton: buffers kept overflowing");
}

}  // namespace

namespace {
int create_impl(const lcs_scene_desc* d, int flags, lcs_stream stream, bool batch, lcs_newton** out);

// the element arrays the selected cloth models need
int check_models(const lcs_scene_desc& d)
{
    if (d.stretch_model != LCS_STRETCH_SPRING && d.stretch_model != LCS_STRETCH_BW98)
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton: unknown stretch model");
    if (d.bending_model != LCS_BENDING_NONE && d.bending_model != LCS_BENDING_QUADRATIC &&
        d.bending_model != LCS_BENDING_DIHEDRAL)
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton: unknown bending model");
    if (d.stretch_model == LCS_STRETCH_BW98 && d.n_stretch_faces &&
        (!d.stretch_faces || !d.stretch_dm_inv || !d.stretch_area))
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton: BW98 stretch needs stretch_faces, stretch_dm_inv, stretch_area");
    if (d.n_bending && !d.bending) return lcs_fail(LCS_ERR_INVALID, "lcs_newton: bending stencils missing");
    if (d.n_bending && d.bending_model == LCS_BENDING_QUADRATIC && !d.bending_Q)
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton: quadratic bending needs bending_Q");
    if (d.n_bending && d.bending_model == LCS_BENDING_DIHEDRAL && (!d.bending_rest_angle || !d.bending_hbar))
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton: dihedral bending needs bending_rest_angle and bending_hbar");
    if (d.n_bodies) {
        if (!d.body || !d.body_dof || !d.body_mass || !d.body_volume || !d.body_kappa || !d.model_x || !d.d_hat)
            return lcs_fail(LCS_ERR_INVALID, "lcs_newton: affine bodies need body, body_dof, body_mass, body_volume, "
                                             "body_kappa and model_x");
        for (uint32_t bi = 0; bi < d.n_bodies; ++bi) {
            const uint32_t s0 = d.body_dof[bi];
            if ((uint64_t)s0 + 4 > d.n_verts) return lcs_fail(LCS_ERR_INVALID, "lcs_newton: body_dof out of range");
            for (uint32_t j = 0; j < 4; ++j)
                if (d.body[s0 + j] != bi || !(d.d_hat[s0 + j] < 0.0f))
                    return lcs_fail(LCS_ERR_INVALID, "lcs_newton: a DOF slot must carry its body id and a negative d_hat");
        }
        for (uint32_t v = 0; v < d.n_verts; ++v)
            if (d.body[v] != kInvalid && d.body[v] >= d.n_bodies)
                return lcs_fail(LCS_ERR_INVALID, "lcs_newton: body id out of range");
    }
    return LCS_OK;
}
}

extern "C" int lcs_newton_create(const lcs_scene_desc* d, int flags, lcs_stream stream, lcs_newton** out)
{
    return create_impl(d, flags, stream, false, out);
}

namespace {
int create_impl(const lcs_scene_desc* d, int flags, lcs_stream stream, bool batch, lcs_newton** out)
{
    if (!d || !out || !d->x || !d->faces || !d->edges || !d->mass || !d->d_hat || !d->offset || !d->vert_area ||
        !d->face_area || !d->edge_area || d->n_verts == 0 || (d->n_edges && !d->rest_len))
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create: incomplete scene description");
    if (int rc = check_models(*d)) return rc;
    lcs_newton* h = new (std::nothrow) lcs_newton();
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create: out of host memory");
    h->d = *d;
    h->flags = flags;
    h->plain = (flags & LCS_NEWTON_PLAIN) != 0;
    h->fp64 = (flags & LCS_NEWTON_FP64) != 0;
    h->profile = (flags & LCS_NEWTON_PROFILE) != 0;
    h->cg1 = (flags & LCS_NEWTON_PCG_SINGLE_REDUCTION) != 0;
    h->full_traversal = (flags & LCS_NEWTON_FULL_TRAVERSAL) != 0;
    h->energy_ls = (flags & LCS_NEWTON_ENERGY_LINESEARCH) != 0;
    h->global_matrix = (flags & LCS_NEWTON_PCG_GLOBAL_MATRIX) != 0;
    h->det = (flags & LCS_NEWTON_DETERMINISTIC) != 0;
    h->batch = batch;
    if (h->det && (d->n_bodies || h->energy_ls || h->plain || d->n_verts >= (1u << 21))) {
        delete h;
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create: LCS_NEWTON_DETERMINISTIC covers fused cloth scenes below "
                                         "2^21 vertices without affine bodies or the energy line search");
    }
    h->V = d->n_verts;
    h->F = d->n_faces;
    h->E = d->n_edges;
    h->B = d->n_bending;
    if (stream) {
        h->s = (cudaStream_t)stream;
    } else {
        cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking);
        h->own_stream = true;
    }
    const size_t V = h->V;
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(upload(h->faces, reinterpret_cast<const uint4*>(d->faces), h->F));
    A(upload(h->edges, reinterpret_cast<const uint2*>(d->edges), h->E));
    A(upload(h->bend, reinterpret_cast<const uint4*>(d->bending), h->B));
    if (d->bending_model == LCS_BENDING_QUADRATIC) A(upload(h->Q, d->bending_Q, 16 * (size_t)h->B));
    if (d->bending_model == LCS_BENDING_DIHEDRAL) {
        A(upload(h->rest_angle, d->bending_rest_angle, h->B));
        A(upload(h->hbar, d->bending_hbar, h->B));
    }
    if (d->n_bodies) {
        h->NB = d->n_bodies;
        std::vector<int8_t> slot(V, -1);
        std::vector<uint8_t> fixed(h->NB, 0);
        for (uint32_t bi = 0; bi < h->NB; ++bi)
            for (uint32_t j = 0; j < 4; ++j) slot[d->body_dof[bi] + j] = (int8_t)j;
        for (size_t v = 0; v < V; ++v)
            if (d->body[v] != kInvalid && slot[v] < 0 && d->pinned && d->pinned[v]) fixed[d->body[v]] = 1;
        A(upload(h->body_dof, d->body_dof, h->NB));
        A(upload(h->bmass, d->body_mass, 16 * (size_t)h->NB));
        A(upload(h->bvol, d->body_volume, h->NB));
        A(upload(h->bkappa, d->body_kappa, h->NB));
        A(upload(h->bfixed, fixed.data(), h->NB));
        A(upload(h->model_x, reinterpret_cast<const float4*>(d->model_x), V));
        A(upload(h->slot, slot.data(), V));
    }
    if (d->stretch_model == LCS_STRETCH_BW98 && d->stretch_mu_lambda)
        A(upload(h->ml, reinterpret_cast<const float2*>(d->stretch_mu_lambda), d->n_stretch_faces));
    if (d->bending_model == LCS_BENDING_DIHEDRAL && d->bending_stiffness) A(upload(h->bend_kper, d->bending_stiffness, h->B));
    if (d->stretch_model == LCS_STRETCH_SPRING && d->spring_stiffness) A(upload(h->spring_kper, d->spring_stiffness, h->E));
    if (d->stretch_model == LCS_STRETCH_BW98) {
        h->Fs = d->n_stretch_faces;
        A(upload(h->sfaces, reinterpret_cast<const uint4*>(d->stretch_faces), h->Fs));
        A(upload(h->dm, reinterpret_cast<const float4*>(d->stretch_dm_inv), h->Fs));
        A(upload(h->sarea, d->stretch_area, h->Fs));
    }
    A(upload(h->rest_len, d->rest_len, h->E));
    A(upload(h->vert_area, d->vert_area, V));
    A(upload(h->face_area, d->face_area, h->F));
    A(upload(h->edge_area, d->edge_area, h->E));
    A(upload(h->mass, d->mass, V));
    A(upload(h->dhat, d->d_hat, V));
    A(upload(h->offset, d->offset, V));
    // the once-per-pair EE traversal applies when the EE queries' boxes are symmetric
    if (h->E > 0) {
        const float D = d->d_hat[d->edges[0]];
        bool sym = D >= 0.0f;
        for (uint32_t e = 0; e < h->E && sym; ++e) {
            const uint32_t v0 = d->edges[2 * e];
            sym = d->offset[v0] == 0.0f && d->d_hat[v0] == D;
        }
        h->ee_sym = sym;
        h->ee_dhat = D;
    }
    {
        std::vector<uint32_t> body(V, kInvalid);
        if (d->body) std::memcpy(body.data(), d->body, 4 * V);
        A(upload(h->body, body.data(), V));
    }
    if (d->pinned) A(upload(h->pinned, d->pinned, V));
    if (d->anim_group && d->n_anim) {
        A(upload(h->group, d->anim_group, V));
        A(upload(h->anim, reinterpret_cast<const Anim*>(d->anim), d->n_anim));
    }
    A(upload(h->rest, reinterpret_cast<const float4*>(d->x), V));
    A(upload(h->x, reinterpret_cast<const float4*>(d->x), V));
    A(dalloc(h->v, V));
    if (e == cudaSuccess) e = d->v ? cudaMemcpy(h->v, d->v, 16 * V, cudaMemcpyHostToDevice) : cudaMemset(h->v, 0, 16 * V);
    A(dalloc(h->x_step, V));
    A(dalloc(h->x_iter, V));
    A(dalloc(h->x_tilde, V));
    A(dalloc(h->target, V));
    A(dalloc(h->dx, V));
    A(dalloc(h->b, V));
    A(dalloc(h->diag, 3 * V));
    A(dalloc(h->st, 1));
    A(dalloc(h->prev_ccd, 2));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_st), sizeof(Status));
    if (h->energy_ls) {
        A(dalloc(h->ls_E, kLsSlots));
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_ls_E), sizeof(double) * kLsSlots);
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_alpha), sizeof(float));
    }
    if (h->plain) {
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_x), 16 * V);
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_v), 16 * V);
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_x_iter), 16 * V);
        if (e == cudaSuccess) std::memcpy(h->h_x, d->x, 16 * V);
        if (e == cudaSuccess) {
            if (d->v) std::memcpy(h->h_v, d->v, 16 * V);
            else std::memset(h->h_v, 0, 16 * V);
        }
    }
    if (e != cudaSuccess) {
        lcs_newton_destroy(h);
        return lcs_fail(LCS_ERR_CUDA, "lcs_newton_create: allocation failed");
    }
    std::memset(h->h_st, 0, sizeof(Status));
    int rc;
    h->sell = !h->plain && !h->batch && (int64_t)h->V <= lcs_pcg_rows_capacity();
    if ((rc = build_material_pattern(h, d)) ||
        (!h->batch && (rc = lcs_bvh_create(LCS_TREE_FACE, h->F, &h->face_tree))) ||
        (!h->batch && (rc = lcs_bvh_create(LCS_TREE_EDGE, h->E, &h->edge_tree))) || (rc = lcs_pcg_create(h->V, &h->pcg))) {
        lcs_newton_destroy(h);
        return rc;
    }
    // CollisionData::resize_collision_data_list (collision_data.h:445-485)
    h->cap_vf = std::max<uint32_t>(4 * h->V, 1024);
    h->cap_ee = std::max<uint32_t>(4 * h->E, 1024);
    h->cap_pairs = std::max<uint32_t>(2 * (h->V + h->E), 1024);
    if ((rc = alloc_contact(h))) {
        lcs_newton_destroy(h);
        return rc;
    }
    if (h->profile)
        for (auto& ev : h->ev) cudaEventCreate(&ev);
    if (!h->plain && (cudaStreamCreateWithFlags(&h->s2, cudaStreamNonBlocking) != cudaSuccess ||
                      cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming) != cudaSuccess ||
                      cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming) != cudaSuccess ||
                      cudaStreamCreateWithFlags(&h->s3, cudaStreamNonBlocking) != cudaSuccess ||
                      cudaEventCreateWithFlags(&h->fork_m, cudaEventDisableTiming) != cudaSuccess ||
                      cudaEventCreateWithFlags(&h->join_m, cudaEventDisableTiming) != cudaSuccess)) {
        lcs_newton_destroy(h);
        return lcs_fail(LCS_ERR_CUDA, "lcs_newton_create: stream/event creation failed");
    }
    *out = h;
    return LCS_OK;
}
}  // namespace

extern "C" int lcs_newton_create_batch(const lcs_scene_desc* descs, uint32_t n_scenes, int flags, lcs_stream stream,
                                       int pcg_cluster, lcs_newton** out)
{
    if (!descs || !out || n_scenes == 0) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: bad argument");
    if (flags & LCS_NEWTON_PLAIN) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: the batch runs fused only");
    if (flags & LCS_NEWTON_ENERGY_LINESEARCH)
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: the energy line search runs on single scenes only");
    if (pcg_cluster != 0 && pcg_cluster != 1 && pcg_cluster != 2 && pcg_cluster != 4 && pcg_cluster != 8 &&
        pcg_cluster != 16)
        return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: cluster size must be 0 (auto), 1, 2, 4, 8 or 16");
    const lcs_scene_desc& d0 = descs[0];
    // concatenate the scenes: indices shifted by the vertex offset, animation groups renumbered
    std::vector<uint32_t> voff(n_scenes + 1, 0), foff(n_scenes + 1, 0), eoff(n_scenes + 1, 0), boff(n_scenes + 1, 0),
        soff(n_scenes + 1, 0), aoff(n_scenes + 1, 0);
    uint32_t groups = 0;
    for (uint32_t s = 0; s < n_scenes; ++s) {
        const lcs_scene_desc& d = descs[s];
        if (!d.x || !d.faces || !d.edges || !d.mass || !d.d_hat || !d.offset || !d.vert_area || !d.face_area ||
            !d.edge_area || d.n_verts == 0 || d.n_faces < 2 || d.n_edges < 2 || !d.rest_len)
            return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: incomplete scene description");
        if (int rc = check_models(d)) return rc;
        if (d.stretch_model != d0.stretch_model || d.bending_model != d0.bending_model ||
            d.stretch_mu != d0.stretch_mu || d.stretch_lambda != d0.stretch_lambda ||
            d.bending_scaling != d0.bending_scaling)
            return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: scenes must share the cloth models and parameters");
        if (d.dt != d0.dt || d.gravity[0] != d0.gravity[0] || d.gravity[1] != d0.gravity[1] ||
            d.gravity[2] != d0.gravity[2] || d.kappa != d0.kappa || d.spring_k != d0.spring_k ||
            d.bending_k != d0.bending_k || d.dirichlet != d0.dirichlet || d.damping != d0.damping ||
            d.nonlinear_iters != d0.nonlinear_iters || d.pcg_max_iter != d0.pcg_max_iter ||
            d.pcg_rel_tol != d0.pcg_rel_tol || d.pcg_abs_rz_tol != d0.pcg_abs_rz_tol || d.use_floor)
            return lcs_fail(LCS_ERR_INVALID,
                            "lcs_newton_create_batch: scenes must share dt, gravity, stiffnesses and solver settings (floor off)");
        voff[s + 1] = voff[s] + d.n_verts;
        foff[s + 1] = foff[s] + d.n_faces;
        eoff[s + 1] = eoff[s] + d.n_edges;
        boff[s + 1] = boff[s] + d.n_bending;
        soff[s + 1] = soff[s] + (d.stretch_model == LCS_STRETCH_BW98 ? d.n_stretch_faces : 0);
        aoff[s + 1] = aoff[s] + d.n_bodies;
        groups += d.anim_group ? d.n_anim : 0;
    }
    if (groups > 127) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: more than 127 animation groups");
    const uint32_t V = voff[n_scenes], F = foff[n_scenes], E = eoff[n_scenes], B = boff[n_scenes], Fs = soff[n_scenes];
    const bool quad = d0.bending_model == LCS_BENDING_QUADRATIC, dih = d0.bending_model == LCS_BENDING_DIHEDRAL;
    std::vector<uint32_t> sfaces(4 * (size_t)Fs);
    std::vector<float> dm(4 * (size_t)Fs), sarea(Fs), rest_angle(dih ? B : 0), hbar(dih ? B : 0);
    const uint32_t NBt = aoff[n_scenes];
    const bool has_ml = d0.stretch_mu_lambda != nullptr, has_bk = d0.bending_stiffness != nullptr,
               has_sk = d0.spring_stiffness != nullptr;
    std::vector<float> mlv(has_ml ? 2 * (size_t)Fs : 0), bkv(has_bk ? B : 0), skv(has_sk ? E : 0);
    std::vector<uint32_t> body_dof(NBt);
    std::vector<float> bmass(16 * (size_t)NBt), bvol(NBt), bkappa(NBt), model_x(NBt ? 4 * (size_t)V : 0, 0.0f);
    std::vector<float> x(4 * (size_t)V), v(4 * (size_t)V, 0.0f), Q(quad ? 16 * (size_t)B : 0), rest_len(E), vert_area(V),
        face_area(F), edge_area(E), mass(V), dhat(V), offset(V), anim(16 * (size_t)std::max(groups, 1u), 0.0f);
    std::vector<uint32_t> faces(4 * (size_t)F), edges(2 * (size_t)E), bend(4 * (size_t)B), body(V, kInvalid);
    std::vector<uint8_t> pinned(V, 0);
    std::vector<int8_t> group(V, -1);
    uint32_t g0 = 0;
    for (uint32_t s = 0; s < n_scenes; ++s) {
        const lcs_scene_desc& d = descs[s];
        const uint32_t vo = voff[s];
        std::memcpy(&x[4 * (size_t)vo], d.x, 16 * (size_t)d.n_verts);
        if (d.v) std::memcpy(&v[4 * (size_t)vo], d.v, 16 * (size_t)d.n_verts);
        for (size_t k = 0; k < 4 * (size_t)d.n_faces; ++k)
            faces[4 * (size_t)foff[s] + k] = (k % 4 == 3) ? d.faces[k] : d.faces[k] + vo;
        for (size_t k = 0; k < 2 * (size_t)d.n_edges; ++k) edges[2 * (size_t)eoff[s] + k] = d.edges[k] + vo;
        for (size_t k = 0; k < 4 * (size_t)d.n_bending; ++k) bend[4 * (size_t)boff[s] + k] = d.bending[k] + vo;
        if (d.n_bending && quad) std::memcpy(&Q[16 * (size_t)boff[s]], d.bending_Q, 64 * (size_t)d.n_bending);
        if (d.n_bending && dih) {
            std::memcpy(&rest_angle[boff[s]], d.bending_rest_angle, 4 * (size_t)d.n_bending);
            std::memcpy(&hbar[boff[s]], d.bending_hbar, 4 * (size_t)d.n_bending);
        }
        const uint32_t ns = soff[s + 1] - soff[s];
        for (size_t k = 0; k < 4 * (size_t)ns; ++k)
            sfaces[4 * (size_t)soff[s] + k] = (k % 4 == 3) ? d.stretch_faces[k] : d.stretch_faces[k] + vo;
        if (ns) {
            std::memcpy(&dm[4 * (size_t)soff[s]], d.stretch_dm_inv, 16 * (size_t)ns);
            std::memcpy(&sarea[soff[s]], d.stretch_area, 4 * (size_t)ns);
        }
        std::memcpy(&rest_len[eoff[s]], d.rest_len, 4 * (size_t)d.n_edges);
        std::memcpy(&vert_area[vo], d.vert_area, 4 * (size_t)d.n_verts);
        std::memcpy(&face_area[foff[s]], d.face_area, 4 * (size_t)d.n_faces);
        std::memcpy(&edge_area[eoff[s]], d.edge_area, 4 * (size_t)d.n_edges);
        std::memcpy(&mass[vo], d.mass, 4 * (size_t)d.n_verts);
        std::memcpy(&dhat[vo], d.d_hat, 4 * (size_t)d.n_verts);
        std::memcpy(&offset[vo], d.offset, 4 * (size_t)d.n_verts);
        if (d.body)
            for (uint32_t k = 0; k < d.n_verts; ++k)
                body[vo + k] = d.body[k] == kInvalid ? kInvalid : d.body[k] + aoff[s];
        for (uint32_t k = 0; k < d.n_bodies; ++k) {
            body_dof[aoff[s] + k] = d.body_dof[k] + vo;
            std::memcpy(&bmass[16 * (size_t)(aoff[s] + k)], d.body_mass + 16 * (size_t)k, 64);
            bvol[aoff[s] + k] = d.body_volume[k];
            bkappa[aoff[s] + k] = d.body_kappa[k];
        }
        if (d.n_bodies) std::memcpy(&model_x[4 * (size_t)vo], d.model_x, 16 * (size_t)d.n_verts);
        if ((d.stretch_mu_lambda != nullptr) != has_ml || (d.bending_stiffness != nullptr) != has_bk ||
            (d.spring_stiffness != nullptr) != has_sk)
            return lcs_fail(LCS_ERR_INVALID, "lcs_newton_create_batch: per-element material arrays given for some scenes only");
        if (has_ml && ns) std::memcpy(&mlv[2 * (size_t)soff[s]], d.stretch_mu_lambda, 8 * (size_t)ns);
        if (has_bk && d.n_bending) std::memcpy(&bkv[boff[s]], d.bending_stiffness, 4 * (size_t)d.n_bending);
        if (has_sk) std::memcpy(&skv[eoff[s]], d.spring_stiffness, 4 * (size_t)d.n_edges);
        if (d.pinned) std::memcpy(&pinned[vo], d.pinned, d.n_verts);
        if (d.anim_group && d.n_anim) {
            for (uint32_t k = 0; k < d.n_verts; ++k)
                group[vo + k] = d.anim_group[k] >= 0 ? (int8_t)(d.anim_group[k] + (int)g0) : (int8_t)-1;
            std::memcpy(&anim[16 * (size_t)g0], d.anim, 64 * (size_t)d.n_anim);
            g0 += d.n_anim;
        }
    }
    lcs_scene_desc D = d0;
    D.n_verts = V; D.n_faces = F; D.n_edges = E; D.n_bending = B;
    D.x = x.data(); D.v = v.data(); D.faces = faces.data(); D.edges = edges.data(); D.bending = bend.data();
    D.bending_Q = Q.data(); D.rest_len = rest_len.data(); D.vert_area = vert_area.data();
    D.n_stretch_faces = Fs; D.stretch_faces = sfaces.data(); D.stretch_dm_inv = dm.data(); D.stretch_area = sarea.data();
    D.bending_rest_angle = rest_angle.data(); D.bending_hbar = hbar.data();
    D.n_bodies = NBt; D.body_dof = body_dof.data(); D.body_mass = bmass.data(); D.body_volume = bvol.data();
    D.body_kappa = bkappa.data(); D.model_x = NBt ? model_x.data() : nullptr;
    D.stretch_mu_lambda = has_ml ? mlv.data() : nullptr; D.bending_stiffness = has_bk ? bkv.data() : nullptr;
    D.spring_stiffness = has_sk ? skv.data() : nullptr;
    D.face_area = face_area.data(); D.edge_area = edge_area.data(); D.mass = mass.data(); D.d_hat = dhat.data();
    D.offset = offset.data(); D.body = body.data(); D.pinned = pinned.data();
    D.anim_group = groups ? group.data() : nullptr; D.n_anim = groups; D.anim = groups ? anim.data() : nullptr;
    lcs_newton* h = nullptr;
    int rc = create_impl(&D, flags, stream, true, &h);
    if (rc) return rc;
    h->S = n_scenes;
    h->cluster = pcg_cluster;
    h->h_voff = voff;
    h->h_foff = foff;
    h->h_eoff = eoff;
    h->sc_iters.assign(n_scenes, 0);
    h->sc_pcg.assign(n_scenes, 0);
    h->sc_toi.assign(n_scenes, 1.0f);
    h->sc_rel.assign(n_scenes, 0.0f);
    h->sc_done.assign(n_scenes, 0);
    std::vector<uint32_t> vscene(V);
    for (uint32_t s = 0; s < n_scenes; ++s) std::fill(vscene.begin() + voff[s], vscene.begin() + voff[s + 1], s);
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(upload(h->vscene, vscene.data(), V));
    {
        bool any = false;
        std::vector<uint8_t> rsv(V, 0);
        for (uint32_t s = 0; s < n_scenes; ++s)
            if (descs[s].n_bodies > 0) {
                any = true;
                std::fill(rsv.begin() + voff[s], rsv.begin() + voff[s + 1], (uint8_t)1);
            }
        if (any) A(upload(h->rigid_scene_v, rsv.data(), V));
    }
    A(upload(h->voff_d, voff.data(), n_scenes + 1));
    A(dalloc(h->active, n_scenes));
    A(dalloc(h->bsc, 3 * (size_t)n_scenes));
    A(dalloc(h->bpcg, n_scenes));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_active), 4 * (size_t)n_scenes);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_bsc), 12 * (size_t)n_scenes);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&h->h_bpcg), sizeof(lcs_pcg_stats) * n_scenes);
    if (e != cudaSuccess) {
        lcs_newton_destroy(h);
        return lcs_fail(LCS_ERR_CUDA, "lcs_newton_create_batch: allocation failed");
    }
    if ((rc = lcs_forest_create(LCS_TREE_FACE, n_scenes, foff.data(), voff.data(), &h->face_forest)) ||
        (rc = lcs_forest_create(LCS_TREE_EDGE, n_scenes, eoff.data(), voff.data(), &h->edge_forest))) {
        lcs_newton_destroy(h);
        return rc;
    }
    *out = h;
    return LCS_OK;
}

extern "C" uint32_t lcs_newton_num_scenes(const lcs_newton* h) { return h ? h->S : 0; }

extern "C" int lcs_newton_scene_stats(const lcs_newton* h, uint32_t scene, lcs_newton_stats* stats)
{
    if (!h || !stats || scene >= h->S) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_scene_stats: bad argument");
    *stats = lcs_newton_stats{};
    if (!h->batch) {
        stats->newton_iters = (int32_t)h->total_newton;
        stats->status = LCS_OK;
        return LCS_OK;
    }
    stats->newton_iters = h->sc_iters[scene];
    stats->pcg_iters = h->sc_pcg[scene];
    stats->last_toi = h->sc_toi[scene];
    stats->last_rel_residual = h->sc_rel[scene];
    stats->status = LCS_OK;
    return LCS_OK;
}

extern "C" int lcs_newton_download_scene(const lcs_newton* h, uint32_t scene, float* x_out, float* v_out)
{
    if (!h || scene >= h->S) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_download_scene: bad argument");
    const uint32_t v0 = h->batch ? h->h_voff[scene] : 0, nv = h->batch ? h->h_voff[scene + 1] - v0 : h->V;
    const size_t bytes = 16 * (size_t)nv;
    if (x_out) LCS_CUDA_TRY(cudaMemcpyAsync(x_out, h->x + v0, bytes, cudaMemcpyDeviceToHost, h->s));
    if (v_out) LCS_CUDA_TRY(cudaMemcpyAsync(v_out, h->v + v0, bytes, cudaMemcpyDeviceToHost, h->s));
    LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    return LCS_OK;
}

extern "C" int lcs_newton_last_iterate(const lcs_newton* h, float* x_iter_out, float* dx_out, float* x_tilde_out)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_last_iterate: null handle");
    const size_t bytes = 16 * (size_t)h->V;
    if (x_iter_out) LCS_CUDA_TRY(cudaMemcpyAsync(x_iter_out, h->x_iter, bytes, cudaMemcpyDeviceToHost, h->s));
    if (dx_out) LCS_CUDA_TRY(cudaMemcpyAsync(dx_out, h->dx, bytes, cudaMemcpyDeviceToHost, h->s));
    if (x_tilde_out) LCS_CUDA_TRY(cudaMemcpyAsync(x_tilde_out, h->x_tilde, bytes, cudaMemcpyDeviceToHost, h->s));
    LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    return LCS_OK;
}

extern "C" int lcs_newton_destroy(lcs_newton* h)
{
    if (!h) return LCS_OK;
    if (h->s) cudaStreamSynchronize(h->s);
    free_contact(h);
    lcs_bvh_destroy(h->face_tree);
    lcs_bvh_destroy(h->edge_tree);
    lcs_forest_destroy(h->face_forest);
    lcs_forest_destroy(h->edge_forest);
    lcs_pcg_destroy(h->pcg);
    {
        void* bp[] = {h->vscene, h->voff_d, h->active, h->bsc, h->bpcg, h->rigid_scene_v};
        for (void* p : bp)
            if (p) cudaFree(p);
        if (h->h_active) cudaFreeHost(h->h_active);
        if (h->h_bsc) cudaFreeHost(h->h_bsc);
        if (h->h_bpcg) cudaFreeHost(h->h_bpcg);
    }
    void* ptrs[] = {h->faces, h->edges, h->bend, h->sfaces, h->dm, h->sarea, h->rest_angle, h->hbar, h->face_slots,
                    h->body_dof, h->bmass, h->bvol, h->bkappa, h->bfixed, h->model_x, h->slot, h->body_slots,
                    h->ml, h->bend_kper, h->spring_kper,
                    h->Q, h->rest_len, h->vert_area, h->face_area, h->edge_area,
                    h->mass, h->dhat, h->offset, h->body, h->pinned, h->group, h->anim, h->rest, h->x, h->v,
                    h->x_step, h->x_iter, h->x_tilde, h->target, h->dx, h->b, h->diag, h->mat_rp, h->mat_col,
                    h->spring_slots, h->bend_slots, h->mat_val, h->st, h->sell_ptr, h->sell_col, h->prev_ccd,
                    h->det_el, h->det_vptr, h->det_bptr, h->det_bbase, h->det_vent, h->det_bent, h->det_n};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->h_st) cudaFreeHost(h->h_st);
    if (h->ls_E) cudaFree(h->ls_E);
    if (h->h_ls_E) cudaFreeHost(h->h_ls_E);
    if (h->h_alpha) cudaFreeHost(h->h_alpha);
    if (h->h_x) cudaFreeHost(h->h_x);
    if (h->h_v) cudaFreeHost(h->h_v);
    if (h->h_x_iter) cudaFreeHost(h->h_x_iter);
    for (auto& ev : h->ev)
        if (ev) cudaEventDestroy(ev);
    if (h->s2) {
        cudaStreamSynchronize(h->s2);
        cudaStreamDestroy(h->s2);
    }
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    if (h->s3) {
        cudaStreamSynchronize(h->s3);
        cudaStreamDestroy(h->s3);
    }
    if (h->fork_m) cudaEventDestroy(h->fork_m);
    if (h->join_m) cudaEventDestroy(h->join_m);
    if (h->own_stream) cudaStreamDestroy(h->s);
    delete h;
    return LCS_OK;
}

extern "C" int lcs_newton_step(lcs_newton* h, lcs_newton_stats* stats)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_step: null handle");
    const lcs_scene_desc& d = h->d;
    const uint32_t V = h->V;
    int rc;
    const auto t_host0 = std::chrono::steady_clock::now();
    h->retries = 0;
    // the positions at the start of this step are the last iterate of the previous one, x_iter + t dx with
    // 0 <= t <= 1, inside that iteration's swept boxes: its CCD lists (element pairs, independent of the
    // trees rebuilt below) filter to this iteration's DCD lists as within a step.  Not across a batch
    // (finished scenes drop out of the last iterations' lists) or after the state was replaced.
    h->filter_ok = h->carry_filter && !h->batch;
    h->carry_filter = false;
    h->time += d.dt;
    h->frame += 1;
    if (h->plain) {  // physics_step_GPU uploads x_step_start, x and v from the host every step
        const size_t bytes = 16 * (size_t)V;
        LCS_CUDA_TRY(cudaMemcpyAsync(h->x_step, h->h_x, bytes, cudaMemcpyHostToDevice, h->s));
        LCS_CUDA_TRY(cudaMemcpyAsync(h->x, h->h_x, bytes, cudaMemcpyHostToDevice, h->s));
        LCS_CUDA_TRY(cudaMemcpyAsync(h->v, h->h_v, bytes, cudaMemcpyHostToDevice, h->s));
        LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    }
    mark(h, kPhBuild);
    k_targets<<<grid256(V), 256, 0, h->s>>>(V, h->rest, h->group, h->anim, (float)h->time, h->target);
    lcs_count_launch();
    k_predict<<<grid256(V), 256, 0, h->s>>>(V, d.dt, d.gravity[0], d.gravity[1], d.gravity[2], h->pinned, h->target, h->x,
                                      h->v, h->x_step, h->x_tilde, abd_of(h));
    lcs_count_launch();
    if (h->NB) {
        k_abd_rigid_tilde<<<grid256(V), 256, 0, h->s>>>(V, abd_of(h), h->x_tilde);
        lcs_count_launch();
    }
    // Init LBVH once per step (newton_solver.cpp:4152-4161)
    const float* XS = reinterpret_cast<const float*>(h->x_step);
    // fused single scene: the edge tree is built on s2 beside the face tree (independent sorts and builds)
    const bool two = !h->batch && !h->plain && h->s2;
    cudaStream_t es = two ? h->s2 : h->s;
    if (two) {
        LCS_CUDA_TRY(cudaEventRecord(h->fork, h->s));
        LCS_CUDA_TRY(cudaStreamWaitEvent(es, h->fork, 0));
    }
    if (!h->batch) {
        if ((rc = lcs_bvh_reduce_aabb(h->face_tree, XS, reinterpret_cast<const uint32_t*>(h->faces), V, h->s))) return rc;
        if ((rc = lcs_bvh_reduce_aabb(h->edge_tree, XS, reinterpret_cast<const uint32_t*>(h->edges), V, es))) return rc;
    }
    if (h->batch) {
        if ((rc = lcs_forest_build(h->face_forest, XS, reinterpret_cast<const uint32_t*>(h->faces), h->s))) return rc;
        if ((rc = lcs_forest_build(h->edge_forest, XS, reinterpret_cast<const uint32_t*>(h->edges), h->s))) return rc;
    } else if (h->plain) {
        if ((rc = lcs_bvh_construct_host_sort(h->face_tree, h->s))) return rc;
        if ((rc = lcs_bvh_construct_host_sort(h->edge_tree, h->s))) return rc;
    } else {
        if ((rc = lcs_bvh_construct(h->face_tree, h->s))) return rc;
        if ((rc = lcs_bvh_construct(h->edge_tree, es))) return rc;
    }
    if (two) {
        LCS_CUDA_TRY(cudaEventRecord(h->join, es));
        LCS_CUDA_TRY(cudaStreamWaitEvent(h->s, h->join, 0));
    }
    if (h->profile) {
        mark(h, kPhMaterial);
        cudaEventSynchronize(h->ev[kPhMaterial]);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, h->ev[kPhBuild], h->ev[kPhMaterial]);
        h->phase_ms[kPhBuild] += ms;
        h->phase_launch_count[kPhBuild] += 1;
    }
    if (h->batch) {  // every scene runs its own Newton loop; finished scenes are switched off
        const uint32_t S = h->S;
        std::fill(h->sc_done.begin(), h->sc_done.end(), 0);
        std::fill(h->sc_iters.begin(), h->sc_iters.end(), 0);
        std::fill(h->sc_pcg.begin(), h->sc_pcg.end(), 0);
        for (uint32_t sc = 0; sc < S; ++sc) h->h_active[sc] = 1u;
        LCS_CUDA_TRY(cudaMemcpyAsync(h->active, h->h_active, 4 * (size_t)S, cudaMemcpyHostToDevice, h->s));
        int iter = 0, pcg_total = 0;
        for (iter = 0; iter < 100; ++iter) {
            bool all = true;
            for (uint32_t sc = 0; sc < S; ++sc) all = all && h->sc_done[sc];
            if (all) break;
            if ((rc = newton_iteration(h))) return rc;
            for (uint32_t sc = 0; sc < S; ++sc) {
                if (h->sc_done[sc]) continue;
                h->sc_iters[sc] += 1;
                h->sc_pcg[sc] += h->h_bpcg[sc].iterations;
                pcg_total += h->h_bpcg[sc].iterations;
                h->sc_toi[sc] = h->h_bsc[sc];
                h->sc_rel[sc] = h->h_bpcg[sc].rel_residual;
                const bool global_converged = h->h_bsc[S + sc] < 1e-2f * d.dt;
                const bool dirichlet_converged = h->h_bsc[2 * S + sc] < 1e-3f;
                if (global_converged || (h->sc_iters[sc] >= d.nonlinear_iters && dirichlet_converged)) {
                    h->sc_done[sc] = 1;
                    h->h_active[sc] = 0u;
                }
            }
            LCS_CUDA_TRY(cudaMemcpyAsync(h->active, h->h_active, 4 * (size_t)S, cudaMemcpyHostToDevice, h->s));
        }
        k_update_velocity<<<grid256(V), 256, 0, h->s>>>(V, d.dt, d.damping, h->x, h->x_step, h->v);
        lcs_count_launch();
        LCS_LAUNCH_CHECK();
        h->total_newton += iter;
        h->total_pcg += pcg_total;
        if (stats) {
            const Status& st = *h->h_st;
            *stats = lcs_newton_stats{};
            stats->newton_iters = iter;
            stats->pcg_iters = pcg_total;
            stats->vf_candidates = st.cnt[0];
            stats->ee_candidates = st.cnt[1];
            stats->contact_pairs = st.cnt[2];
            stats->ccd_vf_candidates = st.cnt[3];
            stats->ccd_ee_candidates = st.cnt[4];
            stats->status = LCS_OK;
            stats->retries = h->retries;
            stats->host_ms =
                std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
        }
        return LCS_OK;
    }
    bool global_converged = false, dirichlet_converged = false;
    int iter = 0, pcg_total = 0;
    h->ls_halvings = 0;
    h->iter_log.clear();
    float last_toi = 1.0f, last_rel = 0.0f;
    for (iter = 0; iter < 100; ++iter) {
        if (global_converged || (iter >= d.nonlinear_iters && dirichlet_converged)) break;
        if ((rc = newton_iteration(h))) return rc;
        const Status& s = *h->h_st;
        h->iter_log.push_back(lcs_newton_iter_record{s.pcg_iters, s.pcg_rel, s.toi, s.max_dx, s.cnt[0], s.cnt[1],
                                                     s.cnt[2], s.cnt[3], s.cnt[4]});
        pcg_total += s.pcg_iters;
        last_toi = s.toi;
        last_rel = s.pcg_rel;
        global_converged = s.max_dx < 1e-2f * d.dt;
        dirichlet_converged = s.dirichlet < 1e-3f;
    }
    h->carry_filter = h->filter_ok && !h->full_traversal;
    k_update_velocity<<<grid256(V), 256, 0, h->s>>>(V, d.dt, d.damping, h->x, h->x_step, h->v);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    if (h->plain) {  // x, v copied back to the host at the end of the step
        const size_t bytes = 16 * (size_t)V;
        LCS_CUDA_TRY(cudaMemcpyAsync(h->h_x, h->x, bytes, cudaMemcpyDeviceToHost, h->s));
        LCS_CUDA_TRY(cudaMemcpyAsync(h->h_v, h->v, bytes, cudaMemcpyDeviceToHost, h->s));
        LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    }
    h->total_newton += iter;
    h->total_pcg += pcg_total;
    if (stats) {
        const Status& s = *h->h_st;
        stats->newton_iters = iter;
        stats->pcg_iters = pcg_total;
        stats->last_toi = last_toi;
        stats->last_rel_residual = last_rel;
        stats->last_alpha = h->last_alpha;
        stats->ls_halvings = h->ls_halvings;
        stats->vf_candidates = s.cnt[0];
        stats->ee_candidates = s.cnt[1];
        stats->contact_pairs = s.cnt[2];
        stats->ccd_vf_candidates = s.cnt[3];
        stats->ccd_ee_candidates = s.cnt[4];
        stats->status = LCS_OK;
        stats->retries = h->retries;
        stats->host_ms =
            std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
    }
    return LCS_OK;
}

extern "C" int lcs_newton_iteration_log(const lcs_newton* h, lcs_newton_iter_record* out, int32_t cap,
                                        int32_t* n_out)
{
    if (!h || !n_out || (cap > 0 && !out)) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_iteration_log: null argument");
    const int32_t n = (int32_t)h->iter_log.size();
    for (int32_t k = 0; k < n && k < cap; ++k) out[k] = h->iter_log[k];
    *n_out = n;
    return LCS_OK;
}

extern "C" int lcs_newton_step_host(lcs_newton* h, const float* x_in, const float* v_in, float* x_out, float* v_out,
                                    lcs_newton_stats* stats)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_step_host: null handle");
    const size_t bytes = 16 * (size_t)h->V;
    if (x_in) h->carry_filter = false;  // new positions: no CCD list describes them
    if (x_in) LCS_CUDA_TRY(cudaMemcpyAsync(h->x, x_in, bytes, cudaMemcpyHostToDevice, h->s));
    if (v_in) LCS_CUDA_TRY(cudaMemcpyAsync(h->v, v_in, bytes, cudaMemcpyHostToDevice, h->s));
    if (h->plain) {
        if (x_in) std::memcpy(h->h_x, x_in, bytes);
        if (v_in) std::memcpy(h->h_v, v_in, bytes);
    }
    int rc = lcs_newton_step(h, stats);
    if (rc) return rc;
    if (x_out) LCS_CUDA_TRY(cudaMemcpyAsync(x_out, h->x, bytes, cudaMemcpyDeviceToHost, h->s));
    if (v_out) LCS_CUDA_TRY(cudaMemcpyAsync(v_out, h->v, bytes, cudaMemcpyDeviceToHost, h->s));
    LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    return LCS_OK;
}

extern "C" int lcs_newton_download(const lcs_newton* h, float* x_out, float* v_out)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_download: null handle");
    const size_t bytes = 16 * (size_t)h->V;
    if (x_out) LCS_CUDA_TRY(cudaMemcpyAsync(x_out, h->x, bytes, cudaMemcpyDeviceToHost, h->s));
    if (v_out) LCS_CUDA_TRY(cudaMemcpyAsync(v_out, h->v, bytes, cudaMemcpyDeviceToHost, h->s));
    LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    return LCS_OK;
}

// SolverInterface::load_saved_state_from_host (solver_interface.cpp:275-412) followed by the upload of the
// frame state: the next step starts from these positions / velocities.
extern "C" int lcs_newton_upload(lcs_newton* h, const float* x_in, const float* v_in)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_upload: null handle");
    const size_t bytes = 16 * (size_t)h->V;
    if (x_in) h->carry_filter = false;
    if (x_in) LCS_CUDA_TRY(cudaMemcpyAsync(h->x, x_in, bytes, cudaMemcpyHostToDevice, h->s));
    if (v_in) LCS_CUDA_TRY(cudaMemcpyAsync(h->v, v_in, bytes, cudaMemcpyHostToDevice, h->s));
    if (h->plain) {
        if (x_in) std::memcpy(h->h_x, x_in, bytes);
        if (v_in) std::memcpy(h->h_v, v_in, bytes);
    }
    LCS_CUDA_TRY(cudaStreamSynchronize(h->s));
    return LCS_OK;
}

extern "C" int lcs_newton_invalidate(lcs_newton* h)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_invalidate: null handle");
    h->carry_filter = false;
    return LCS_OK;
}

extern "C" int lcs_newton_set_frame(lcs_newton* h, uint32_t frame)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_set_frame: null handle");
    h->frame = frame;
    h->time = (double)frame * (double)h->d.dt;
    return LCS_OK;
}

extern "C" int lcs_newton_get_frame(const lcs_newton* h, uint32_t* frame_out)
{
    if (!h || !frame_out) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_get_frame: null argument");
    *frame_out = h->frame;
    return LCS_OK;
}

extern "C" int lcs_newton_state(const lcs_newton* h, float** d_x, float** d_v)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_state: null handle");
    if (d_x) *d_x = reinterpret_cast<float*>(h->x);
    if (d_v) *d_v = reinterpret_cast<float*>(h->v);
    return LCS_OK;
}

extern "C" int lcs_newton_profile(const lcs_newton* h, double* phase_ms, int32_t* launches, int n)
{
    if (!h || !phase_ms) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_profile: bad argument");
    for (int p = 0; p < n && p < kPhases; ++p) {
        phase_ms[p] = h->phase_ms[p];
        if (launches) launches[p] = h->phase_launch_count[p];
    }
    return LCS_OK;
}

extern "C" int lcs_newton_reset_profile(lcs_newton* h)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_reset_profile: null handle");
    for (int p = 0; p < kPhases; ++p) {
        h->phase_ms[p] = 0.0;
        h->phase_launch_count[p] = 0;
    }
    return LCS_OK;
}

extern "C" int lcs_newton_batch_query_tuning(const lcs_newton* h, uint32_t* vf_threads, uint32_t* ee_threads)
{
    if (!h || !h->batch) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_batch_query_tuning: needs a batch handle");
    int rc = lcs_forest_query_tuning(h->face_forest, vf_threads, nullptr);
    if (rc == LCS_OK) rc = lcs_forest_query_tuning(h->edge_forest, ee_threads, nullptr);
    return rc;
}

extern "C" int lcs_newton_batch_tuning(const lcs_newton* h, uint32_t* chunks_per_cta, float* solve_ms)
{
    if (!h || !h->pcg) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_batch_tuning: bad handle");
    return lcs_pcg_batch_tuning(h->pcg, chunks_per_cta, solve_ms);
}

extern "C" int lcs_newton_pcg_kind(const lcs_newton* h)
{
    if (!h) return -1;
    if (h->plain) return 0;
    if (!h->sell) return 1;
    if (!h->cg1) return 2;
    return !h->global_matrix && lcs_pcg_resident(h->pcg) ? 4 : 3;
}

extern "C" int lcs_newton_counts(const lcs_newton* h, uint32_t* nnz_material, uint32_t* cap_vf, uint32_t* cap_ee,
                                 uint32_t* cap_pairs)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_newton_counts: null handle");
    if (nnz_material) *nnz_material = h->nnz_mat;
    if (cap_vf) *cap_vf = h->cap_vf;
    if (cap_ee) *cap_ee = h->cap_ee;
    if (cap_pairs) *cap_pairs = h->cap_pairs;
    return LCS_OK;
}
