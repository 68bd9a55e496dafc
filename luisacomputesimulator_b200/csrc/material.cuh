// material.cuh -- the cloth energies the Newton loop assembles besides inertia and contact:
//  * Baraff-Witkin stretch + shear of a triangle (StretchEnergy::compute_gradient_hessian,
//    Solver/Energy/stretch_energy.h:440-476, with detail::stretch_* / shear_* :215-321 and the
//    chain rule convert_force / convert_hessian :156-185), the reference's FEM_BW98 model;
//  * discrete-shell dihedral-angle bending with a Gauss-Newton Hessian (fn_evaluate_bending,
//    Solver/SimulationSolver/newton_solver.cpp:1102-1175, BendingEnergy::compute_d_theta_d_x,
//    Solver/Energy/bending_energy.h:167-263), the model the reference's Newton solver evaluates
//    for every bending model other than None.
//
// The arithmetic is written out term by term (no implicit contraction, -fmad=false) in the order
// the CPU oracle restates it, so both produce the same bits except where acosf is involved.
//
// BW98 in block form.  With F = [Fu Fv] = [x1 - x0, x2 - x0] Dm^-1 (Dm^-1 columns (d0, d1),
// (d2, d3)), vertex a moves F by w_a = (w_a0, w_a1): w_0 = (-(d0 + d1), -(d2 + d3)),
// w_1 = (d0, d2), w_2 = (d1, d3).  The energy gradient is area * (w_a0 dE/dFu + w_a1 dE/dFv)
// and the 3x3 Hessian block (a, b) is area * sum_{c,d} w_ac w_bd H_cd, where H_cd are the 3x3
// blocks of the projected 6x6 Hessian in F (stretch: mu (max(0, 1 - 1/|Fu|) I + min(1/|Fu|, 1)
// fu fu^T) per column; shear: lambda (|I6| (T - Tq Tq^T / |Tq|^2) + lambda0 q0 q0^T) with
// I6 = Fu.Fv, T = (I + sign(I6) S) / 2, S the column swap, q0 the normalised
// I6 [Fu; Fv] + lambda0 [Fv; Fu], lambda0 = (|F|^2 + sqrt(|F|^4 + 12 I6^2)) / 2).  This is the
// same matrix as dF/dx^T H dF/dx of convert_hessian; blocks (b, a) with b > a are the transposes
// of (a, b), so the assembled matrix is symmetric bit for bit.
#pragma once
#include "lcs_common.cuh"

namespace lcs {

__device__ __forceinline__ float sgnf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// 3x3 blocks are stored column-major: element (row r, col c) at [3 * c + r]
struct Bw98Out {
    v3 g[3];          // dE/dx_a
    float K[6][9];    // blocks (0,0) (1,1) (2,2) (0,1) (0,2) (1,2)
};

__device__ __forceinline__ void bw98_face(v3 x0, v3 x1, v3 x2, float4 dm, float mu, float lambda, float area,
                                          Bw98Out& o)
{
    const v3 e1 = x1 - x0, e2 = x2 - x0;
    const v3 Fu = mk3(__fmaf_rn(e2.x, dm.y, e1.x * dm.x), __fmaf_rn(e2.y, dm.y, e1.y * dm.x),
                      __fmaf_rn(e2.z, dm.y, e1.z * dm.x));
    const v3 Fv = mk3(__fmaf_rn(e2.x, dm.w, e1.x * dm.z), __fmaf_rn(e2.y, dm.w, e1.y * dm.z),
                      __fmaf_rn(e2.z, dm.w, e1.z * dm.z));
    const float I5u = dot3(Fu, Fu), I5v = dot3(Fv, Fv), I6 = dot3(Fu, Fv);
    const float su = sqrtf(I5u), sv = sqrtf(I5v);
    const float iu = 1.0f / su, iv = 1.0f / sv;
    // dE/dF (stretch + shear)
    const float cu = ((su - 1.0f) * iu) * mu, cv = ((sv - 1.0f) * iv) * mu, sw = lambda * I6;
    const v3 Pu = mk3(__fmaf_rn(sw, Fv.x, cu * Fu.x), __fmaf_rn(sw, Fv.y, cu * Fu.y), __fmaf_rn(sw, Fv.z, cu * Fu.z));
    const v3 Pv = mk3(__fmaf_rn(sw, Fu.x, cv * Fv.x), __fmaf_rn(sw, Fu.y, cv * Fv.y), __fmaf_rn(sw, Fu.z, cv * Fv.z));
    const float w[3][2] = {{-(dm.x + dm.y), -(dm.z + dm.w)}, {dm.x, dm.z}, {dm.y, dm.w}};
#pragma unroll
    for (int a = 0; a < 3; ++a)
        o.g[a] = mk3(area * __fmaf_rn(w[a][1], Pv.x, w[a][0] * Pu.x), area * __fmaf_rn(w[a][1], Pv.y, w[a][0] * Pu.y),
                     area * __fmaf_rn(w[a][1], Pv.z, w[a][0] * Pu.z));
    // projected 6x6 Hessian in F: blocks uu, uv, vv
    const float au = fmx(0.0f, 1.0f - iu), av = fmx(0.0f, 1.0f - iv);
    const float bu = fmn(iu, 1.0f), bv = fmn(iv, 1.0f);
    const v3 fu = iu * Fu, fv = iv * Fv;
    const float sg = sgnf(I6), a6 = fabsf(I6);
    const float I2 = I5u + I5v;
    const float lam0 = 0.5f * (I2 + sqrtf(__fmaf_rn(12.0f * I6, I6, I2 * I2)));
    const v3 qu = mk3(__fmaf_rn(lam0, Fv.x, I6 * Fu.x), __fmaf_rn(lam0, Fv.y, I6 * Fu.y), __fmaf_rn(lam0, Fv.z, I6 * Fu.z));
    const v3 qv = mk3(__fmaf_rn(lam0, Fu.x, I6 * Fv.x), __fmaf_rn(lam0, Fu.y, I6 * Fv.y), __fmaf_rn(lam0, Fu.z, I6 * Fv.z));
    const float nq = sqrtf(dot3(qu, qu) + dot3(qv, qv));
    const float q[6] = {qu.x / nq, qu.y / nq, qu.z / nq, qv.x / nq, qv.y / nq, qv.z / nq};
    float t[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        t[k] = 0.5f * __fmaf_rn(sg, q[3 + k], q[k]);
        t[3 + k] = 0.5f * __fmaf_rn(sg, q[k], q[3 + k]);
    }
    const float nT = dot3(mk3(t[0], t[1], t[2]), mk3(t[0], t[1], t[2])) + dot3(mk3(t[3], t[4], t[5]), mk3(t[3], t[4], t[5]));
    const float fuv[6] = {fu.x, fu.y, fu.z, fv.x, fv.y, fv.z};
    // H(i, j) for i, j in 0..5 (i, j < 3: u block); only uu, uv, vv are needed
    auto H = [&](int i, int j) -> float {
        const bool same = (i % 3) == (j % 3);
        const int bi = i / 3, bj = j / 3;
        float id = 0.0f;  // identity part of T in block (bi, bj)
        if (same) id = (bi == bj) ? 0.5f : 0.5f * sg;
        const float shear = lambda * __fmaf_rn(lam0, q[i] * q[j], a6 * (id - (t[i] * t[j]) / nT));
        if (bi != bj) return shear;
        const float ab = bi == 0 ? au : av, bb = bi == 0 ? bu : bv;
        const float stretch = mu * __fmaf_rn(bb, fuv[i] * fuv[j], same ? ab : 0.0f);
        return stretch + shear;
    };
    float Huu[9], Huv[9], Hvv[9];  // column-major: [3 * c + r]
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            Huu[3 * c + r] = H(r, c);
            Huv[3 * c + r] = H(r, 3 + c);
            Hvv[3 * c + r] = H(3 + r, 3 + c);
        }
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float w00 = w[pa[k]][0] * w[pb[k]][0], w01 = w[pa[k]][0] * w[pb[k]][1];
        const float w10 = w[pa[k]][1] * w[pb[k]][0], w11 = w[pa[k]][1] * w[pb[k]][1];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                float s = w00 * Huu[3 * c + r];
                s = __fmaf_rn(w01, Huv[3 * c + r], s);
                s = __fmaf_rn(w10, Huv[3 * r + c], s);
                s = __fmaf_rn(w11, Hvv[3 * c + r], s);
                o.K[k][3 * c + r] = area * s;
            }
    }
}

// Dihedral angle of the hinge (P0, P1) with wings P2, P3 and its gradient
// (BendingEnergy::detail::face_dihedral_angle / face_dihedral_angle_grad as called by
// compute_d_theta_d_x(x[0], x[1], x[2], x[3])).
__device__ __forceinline__ float dihedral_angle_grad(v3 P0, v3 P1, v3 P2, v3 P3, v3 g[4])
{
    const v3 n1 = cross3(P1 - P2, P0 - P2), n2 = cross3(P0 - P3, P1 - P3);
    const float c = dot3(n1, n2) / sqrtf(dot3(n1, n1) * dot3(n2, n2));
    const float ang = acosf(fmx(-1.0f, fmn(1.0f, c)));
    const float theta = sgnf(dot3(cross3(n2, n1), P1 - P0)) * ang;
    const v3 e0 = P0 - P1, e1 = P2 - P1, e2 = P3 - P1, e3 = P2 - P0, e4 = P3 - P0;
    const v3 m1 = cross3(e0, e1), m2 = cross3(e2, e0);
    const float m1s = dot3(m1, m1), m2s = dot3(m2, m2), l = sqrtf(dot3(e0, e0));
    const float l1 = l * m1s, l2 = l * m2s;
    g[2] = (-l / m1s) * m1;
    g[3] = (-l / m2s) * m2;
    const float a1 = -dot3(e0, e3) / l1, a2 = dot3(e0, e4) / l2;
    const float b1 = dot3(e0, e1) / l1, b2 = dot3(e0, e2) / l2;
    g[1] = mk3(a1 * m1.x - a2 * m2.x, a1 * m1.y - a2 * m2.y, a1 * m1.z - a2 * m2.z);
    g[0] = mk3(b1 * m1.x + b2 * m2.x, b1 * m1.y + b2 * m2.y, b1 * m1.z + b2 * m2.z);
    return theta;
}

}  // namespace lcs
