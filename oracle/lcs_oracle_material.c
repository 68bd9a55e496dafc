/*
 * lcs_oracle_material.c -- CPU restatement of the cloth energies of the Newton loop.
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA material kernels and part of the timed CPU
 * baseline.  The product never links it.
 *
 *   Baraff-Witkin stretch + shear   StretchEnergy::compute_gradient_hessian, compute_energy
 *                                   (Solver/Energy/stretch_energy.h:156-321, 440-520)
 *   dihedral bending                fn_evaluate_bending (Solver/SimulationSolver/newton_solver.cpp:1102-1175),
 *                                   BendingEnergy::detail::face_dihedral_angle(_grad)
 *                                   (Solver/Energy/bending_energy.h:167-273)
 *   springs                         fn_evaluate_spring (newton_solver.cpp:1002-1050)
 *   energies                        fn_calc_energy_* (Solver/SimulationSolver/solver_interface.cpp:505-728)
 *
 * The BW98 Hessian is evaluated block by block: with F = [x1 - x0, x2 - x0] Dm^-1 and
 * w_0 = (-(d0 + d1), -(d2 + d3)), w_1 = (d0, d2), w_2 = (d1, d3) the weights of each vertex on the
 * two columns of F, block (a, b) = area * sum_{c,d} w_ac w_bd H_cd, which is the reference's
 * dF/dx^T H dF/dx (convert_hessian) term by term; tests/test_material_oracle.py checks this form
 * against the reference's matrix form in float64.  Operation order: dot products fma(z, fma(y, x*x)),
 * two-term sums fma(b, t, a*s); the CUDA kernels use the same order, so everything but acosf matches
 * bit for bit.
 */
#include "lcs_oracle.h"

#include <math.h>
#include <string.h>

typedef struct { float x, y, z; } m3;

static inline m3 M3(float x, float y, float z) { m3 r = {x, y, z}; return r; }
static inline m3 msub(m3 a, m3 b) { return M3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline m3 mscl(float s, m3 a) { return M3(s * a.x, s * a.y, s * a.z); }
static inline float mdot(m3 a, m3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
static inline m3 mcrs(m3 a, m3 b) { return M3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float mmax(float a, float b) { return a > b ? a : b; }
static inline float mmin(float a, float b) { return a < b ? a : b; }
static inline float msgn(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
static inline m3 mld(const float* x4, uint32_t i) { return M3(x4[4 * (size_t)i], x4[4 * (size_t)i + 1], x4[4 * (size_t)i + 2]); }

/* F = [x1 - x0, x2 - x0] Dm^-1; dm = {d0, d1, d2, d3}, the columns of Dm^-1 */
static void deformation(m3 x0, m3 x1, m3 x2, const float* dm, m3* Fu, m3* Fv)
{
    m3 e1 = msub(x1, x0), e2 = msub(x2, x0);
    *Fu = M3(fmaf(e2.x, dm[1], e1.x * dm[0]), fmaf(e2.y, dm[1], e1.y * dm[0]), fmaf(e2.z, dm[1], e1.z * dm[0]));
    *Fv = M3(fmaf(e2.x, dm[3], e1.x * dm[2]), fmaf(e2.y, dm[3], e1.y * dm[2]), fmaf(e2.z, dm[3], e1.z * dm[2]));
}

/* g[3][3] = dE/dx_a; K[6][9] = blocks (0,0) (1,1) (2,2) (0,1) (0,2) (1,2), column-major [3 c + r] */
void orc_bw98_face(const float* x0p, const float* x1p, const float* x2p, const float* dm, float mu, float lambda,
                   float area, float* g, float* K)
{
    m3 Fu, Fv;
    deformation(M3(x0p[0], x0p[1], x0p[2]), M3(x1p[0], x1p[1], x1p[2]), M3(x2p[0], x2p[1], x2p[2]), dm, &Fu, &Fv);
    const float I5u = mdot(Fu, Fu), I5v = mdot(Fv, Fv), I6 = mdot(Fu, Fv);
    const float su = sqrtf(I5u), sv = sqrtf(I5v);
    const float iu = 1.0f / su, iv = 1.0f / sv;
    /* detail::stretch_gradient + shear_gradient (stretch_energy.h:238-263) */
    const float cu = ((su - 1.0f) * iu) * mu, cv = ((sv - 1.0f) * iv) * mu, sw = lambda * I6;
    const m3 Pu = M3(fmaf(sw, Fv.x, cu * Fu.x), fmaf(sw, Fv.y, cu * Fu.y), fmaf(sw, Fv.z, cu * Fu.z));
    const m3 Pv = M3(fmaf(sw, Fu.x, cv * Fv.x), fmaf(sw, Fu.y, cv * Fv.y), fmaf(sw, Fu.z, cv * Fv.z));
    const float w[3][2] = {{-(dm[0] + dm[1]), -(dm[2] + dm[3])}, {dm[0], dm[2]}, {dm[1], dm[3]}};
    for (int a = 0; a < 3; ++a) { /* convert_force (stretch_energy.h:156-169) */
        g[3 * a + 0] = area * fmaf(w[a][1], Pv.x, w[a][0] * Pu.x);
        g[3 * a + 1] = area * fmaf(w[a][1], Pv.y, w[a][0] * Pu.y);
        g[3 * a + 2] = area * fmaf(w[a][1], Pv.z, w[a][0] * Pu.z);
    }
    /* detail::stretch_hessian (stretch_energy.h:265-290) */
    const float au = mmax(0.0f, 1.0f - iu), av = mmax(0.0f, 1.0f - iv);
    const float bu = mmin(iu, 1.0f), bv = mmin(iv, 1.0f);
    const m3 fu = mscl(iu, Fu), fv = mscl(iv, Fv);
    /* detail::shear_hessian (stretch_energy.h:292-321) */
    const float sg = msgn(I6), a6 = fabsf(I6);
    const float I2 = I5u + I5v;
    const float lam0 = 0.5f * (I2 + sqrtf(fmaf(12.0f * I6, I6, I2 * I2)));
    const m3 qu = M3(fmaf(lam0, Fv.x, I6 * Fu.x), fmaf(lam0, Fv.y, I6 * Fu.y), fmaf(lam0, Fv.z, I6 * Fu.z));
    const m3 qv = M3(fmaf(lam0, Fu.x, I6 * Fv.x), fmaf(lam0, Fu.y, I6 * Fv.y), fmaf(lam0, Fu.z, I6 * Fv.z));
    const float nq = sqrtf(mdot(qu, qu) + mdot(qv, qv));
    const float q[6] = {qu.x / nq, qu.y / nq, qu.z / nq, qv.x / nq, qv.y / nq, qv.z / nq};
    float t[6];
    for (int k = 0; k < 3; ++k) {
        t[k] = 0.5f * fmaf(sg, q[3 + k], q[k]);
        t[3 + k] = 0.5f * fmaf(sg, q[k], q[3 + k]);
    }
    const float nT = mdot(M3(t[0], t[1], t[2]), M3(t[0], t[1], t[2])) + mdot(M3(t[3], t[4], t[5]), M3(t[3], t[4], t[5]));
    const float fuv[6] = {fu.x, fu.y, fu.z, fv.x, fv.y, fv.z};
    float H6[6][6];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            const int same = (i % 3) == (j % 3), bi = i / 3, bj = j / 3;
            float id = 0.0f;
            if (same) id = (bi == bj) ? 0.5f : 0.5f * sg;
            const float shear = lambda * fmaf(lam0, q[i] * q[j], a6 * (id - (t[i] * t[j]) / nT));
            if (bi != bj) {
                H6[i][j] = shear;
            } else {
                const float ab = bi == 0 ? au : av, bb = bi == 0 ? bu : bv;
                H6[i][j] = mu * fmaf(bb, fuv[i] * fuv[j], same ? ab : 0.0f) + shear;
            }
        }
    static const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < 6; ++k) { /* convert_hessian (stretch_energy.h:170-185), block (pa, pb) */
        const float w00 = w[pa[k]][0] * w[pb[k]][0], w01 = w[pa[k]][0] * w[pb[k]][1];
        const float w10 = w[pa[k]][1] * w[pb[k]][0], w11 = w[pa[k]][1] * w[pb[k]][1];
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) {
                float s = w00 * H6[r][c];
                s = fmaf(w01, H6[r][3 + c], s);
                s = fmaf(w10, H6[c][3 + r], s);
                s = fmaf(w11, H6[3 + r][3 + c], s);
                K[9 * k + 3 * c + r] = area * s;
            }
    }
}

/* dihedral angle of hinge (P0, P1) with wings P2, P3 and its gradient g[4][3]
 * (compute_d_theta_d_x(x[0], x[1], x[2], x[3]), bending_energy.h:255-263) */
float orc_dihedral(const float* p0, const float* p1, const float* p2, const float* p3, float* g)
{
    const m3 P0 = M3(p0[0], p0[1], p0[2]), P1 = M3(p1[0], p1[1], p1[2]);
    const m3 P2 = M3(p2[0], p2[1], p2[2]), P3 = M3(p3[0], p3[1], p3[2]);
    /* face_dihedral_angle(P2, P1, P0, P3) (bending_energy.h:222-231) */
    const m3 n1 = mcrs(msub(P1, P2), msub(P0, P2)), n2 = mcrs(msub(P0, P3), msub(P1, P3));
    const float c = mdot(n1, n2) / sqrtf(mdot(n1, n1) * mdot(n2, n2));
    const float ang = acosf(mmax(-1.0f, mmin(1.0f, c)));
    const float theta = msgn(mdot(mcrs(n2, n1), msub(P1, P0))) * ang;
    /* face_dihedral_angle_grad(v2 = P2, v0 = P1, v1 = P0, v3 = P3) (bending_energy.h:167-190) */
    const m3 e0 = msub(P0, P1), e1 = msub(P2, P1), e2 = msub(P3, P1), e3 = msub(P2, P0), e4 = msub(P3, P0);
    const m3 m1 = mcrs(e0, e1), m2 = mcrs(e2, e0);
    const float m1s = mdot(m1, m1), m2s = mdot(m2, m2), l = sqrtf(mdot(e0, e0));
    const float l1 = l * m1s, l2 = l * m2s;
    const m3 g2 = mscl(-l / m1s, m1), g3 = mscl(-l / m2s, m2);
    const float a1 = -mdot(e0, e3) / l1, a2 = mdot(e0, e4) / l2;
    const float b1 = mdot(e0, e1) / l1, b2 = mdot(e0, e2) / l2;
    const m3 g1 = M3(a1 * m1.x - a2 * m2.x, a1 * m1.y - a2 * m2.y, a1 * m1.z - a2 * m2.z);
    const m3 g0 = M3(b1 * m1.x + b2 * m2.x, b1 * m1.y + b2 * m2.y, b1 * m1.z + b2 * m2.z);
    const m3 gg[4] = {g0, g1, g2, g3};
    for (int i = 0; i < 4; ++i) {
        g[3 * i] = gg[i].x;
        g[3 * i + 1] = gg[i].y;
        g[3 * i + 2] = gg[i].z;
    }
    return theta;
}

/* 3x3 block K (column-major) to a float3x3 record (three float4 columns), transposed if t */
static void put33(float* o, const float* K, int t)
{
    for (int c = 0; c < 3; ++c) {
        for (int r = 0; r < 3; ++r) o[4 * c + r] = t ? K[3 * r + c] : K[3 * c + r];
        o[4 * c + 3] = 0.0f;
    }
}
static void put3(float* o, const float* g)
{
    o[0] = g[0];
    o[1] = g[1];
    o[2] = g[2];
    o[3] = 0.0f;
}

void orc_eval_stretch_faces(uint32_t n, const float* x4, const uint32_t* faces4, const float* dm4, const float* area,
                            const float* mu_lambda2, float* grad4, float* hess12)
{
#pragma omp parallel for schedule(static)
    for (long long fl = 0; fl < (long long)n; ++fl) {
        const size_t f = (size_t)fl;
        const uint32_t* v = faces4 + 4 * f;
        float g[9], K[54];
        orc_bw98_face(x4 + 4 * (size_t)v[0], x4 + 4 * (size_t)v[1], x4 + 4 * (size_t)v[2], dm4 + 4 * f,
                      mu_lambda2[2 * f], mu_lambda2[2 * f + 1], area[f], g, K);
        for (int a = 0; a < 3; ++a) put3(grad4 + 4 * (3 * f + a), g + 3 * a);
        float* h = hess12 + 12 * 9 * f;
        /* (0,0) (1,1) (2,2) (0,1) (0,2) (1,0) (1,2) (2,0) (2,1) */
        const int src[9] = {0, 1, 2, 3, 4, 3, 5, 4, 5}, tr[9] = {0, 0, 0, 0, 0, 1, 0, 1, 1};
        for (int k = 0; k < 9; ++k) put33(h + 12 * k, K + 9 * src[k], tr[k]);
    }
}

void orc_eval_bending(uint32_t n, const float* x4, const uint32_t* st4, const float* rest_angle, const float* hbar,
                      const float* stiffness, float scaling, float* grad4, float* hess12)
{
#pragma omp parallel for schedule(static)
    for (long long sl = 0; sl < (long long)n; ++sl) {
        const size_t s = (size_t)sl;
        const uint32_t* v = st4 + 4 * s;
        float g[12];
        const float theta = orc_dihedral(x4 + 4 * (size_t)v[0], x4 + 4 * (size_t)v[1], x4 + 4 * (size_t)v[2],
                                         x4 + 4 * (size_t)v[3], g);
        const float stiff = stiffness[s] * scaling * hbar[s];
        const float sd = stiff * (theta - rest_angle[s]);
        for (int i = 0; i < 4; ++i) {
            const float gi[3] = {sd * g[3 * i], sd * g[3 * i + 1], sd * g[3 * i + 2]};
            put3(grad4 + 4 * (4 * s + i), gi);
        }
        float* h = hess12 + 12 * 16 * s;
        int k = 4;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                float K[9];
                for (int c = 0; c < 3; ++c)
                    for (int r = 0; r < 3; ++r) K[3 * c + r] = stiff * (g[3 * i + r] * g[3 * j + c]);
                put33(h + 12 * (i == j ? i : k), K, 0);
                if (i != j) ++k;
            }
    }
}

void orc_eval_springs(uint32_t n, const float* x4, const uint32_t* edges2, const float* rest_len,
                      const float* stiffness, float* grad4, float* hess12)
{
#pragma omp parallel for schedule(static)
    for (long long el = 0; el < (long long)n; ++el) {
        const size_t e = (size_t)el;
        const m3 d = msub(mld(x4, edges2[2 * e]), mld(x4, edges2[2 * e + 1]));
        const float l = mmax(sqrtf(mdot(d, d)), 1.19209290E-7f);
        const float k = stiffness[e], L = rest_len[e];
        const float C = l - L, il = 1.0f / l, il2 = il * il;
        const float g[3] = {k * d.x * il * C, k * d.y * il * C, k * d.z * il * C};
        const float ng[3] = {-g[0], -g[1], -g[2]};
        put3(grad4 + 4 * (2 * e), g);
        put3(grad4 + 4 * (2 * e + 1), ng);
        const float a = k * il2, cc = k * mmax(1.0f - L * il, 0.0f);
        const float dd[3] = {d.x, d.y, d.z};
        float H[9], N[9];
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) {
                H[3 * c + r] = a * dd[r] * dd[c] + cc * ((r == c ? 1.0f : 0.0f) - il2 * dd[r] * dd[c]);
                N[3 * c + r] = -H[3 * c + r];
            }
        float* h = hess12 + 12 * 4 * e;
        put33(h, H, 0);
        put33(h + 12, H, 0);
        put33(h + 24, N, 0);
        put33(h + 36, N, 0);
    }
}

/* fn_calc_energy_inertia / _spring / _stretch_face / _bending, each term summed in double */
void orc_material_energy(uint32_t V, const float* x4, const float* xt4, const float* mass, const uint8_t* fixed,
                         float dt, float dirichlet, uint32_t E, const uint32_t* springs2, const float* rest_len,
                         const float* spring_k, uint32_t Fs, const uint32_t* faces4, const float* dm4,
                         const float* area, const float* mu_lambda2, uint32_t B, const uint32_t* st4,
                         const float* rest_angle, const float* hbar, const float* bend_k, float scaling, double* out)
{
    double e0 = 0.0, e1 = 0.0, e2 = 0.0, e3 = 0.0;
    const float h2inv = 1.0f / (dt * dt);
#pragma omp parallel for reduction(+ : e0) schedule(static)
    for (long long il = 0; il < (long long)V; ++il) {
        const m3 d = msub(mld(x4, (uint32_t)il), mld(xt4, (uint32_t)il));
        float en = h2inv * mdot(d, d) * mass[il] / 2.0f;
        if (fixed && fixed[il]) en = dirichlet * en;
        e0 += (double)en;
    }
#pragma omp parallel for reduction(+ : e1) schedule(static)
    for (long long il = 0; il < (long long)E; ++il) {
        const m3 d = msub(mld(x4, springs2[2 * il + 1]), mld(x4, springs2[2 * il]));
        const float C = sqrtf(mdot(d, d)) - rest_len[il];
        e1 += (double)(0.5f * spring_k[il] * C * C);
    }
#pragma omp parallel for reduction(+ : e2) schedule(static)
    for (long long il = 0; il < (long long)Fs; ++il) {
        const uint32_t* v = faces4 + 4 * il;
        m3 Fu, Fv;
        deformation(mld(x4, v[0]), mld(x4, v[1]), mld(x4, v[2]), dm4 + 4 * il, &Fu, &Fv);
        const float su = sqrtf(mdot(Fu, Fu)) - 1.0f, sv = sqrtf(mdot(Fv, Fv)) - 1.0f, i6 = mdot(Fu, Fv);
        const float en = 0.5f * mu_lambda2[2 * il] * (su * su + sv * sv) + 0.5f * mu_lambda2[2 * il + 1] * (i6 * i6);
        e2 += (double)(area[il] * en);
    }
#pragma omp parallel for reduction(+ : e3) schedule(static)
    for (long long il = 0; il < (long long)B; ++il) {
        const uint32_t* v = st4 + 4 * il;
        float g[12];
        const float th = orc_dihedral(x4 + 4 * (size_t)v[0], x4 + 4 * (size_t)v[1], x4 + 4 * (size_t)v[2],
                                      x4 + 4 * (size_t)v[3], g);
        const float d = th - rest_angle[il];
        e3 += (double)(0.5f * bend_k[il] * scaling * hbar[il] * d * d);
    }
    out[0] = e0;
    out[1] = e1;
    out[2] = e2;
    out[3] = e3;
}

/* Inertia + the selected stretch and bending models written into b, the diagonal and the material
 * blocks on a fixed pattern (the fused form of the evaluate + assembly kernels,
 * newton_solver.cpp:705-851, 1002-1175).  stretch_model / bending_model as in lcs_gpu.h; slots:
 * block index of each contribution (springs 2 per edge, faces 6 per face, stencils 12 per stencil). */
void orc_material_fill2(uint32_t V, const float* x4, const float* rest4, const float* xt4, const float* mass,
                        const uint8_t* pinned, float dt, float dirichlet, int stretch_model, int bending_model,
                        uint32_t E, const uint32_t* edges, const float* rest_len, float spring_k, uint32_t Fs,
                        const uint32_t* sfaces4, const float* dm4, const float* sarea, float mu, float lambda,
                        uint32_t B, const uint32_t* stencil, const float* Q16, const float* rest_angle,
                        const float* hbar, float bending_k, float bending_scaling, const uint32_t* spring_slots,
                        const uint32_t* face_slots, const uint32_t* bend_slots, uint32_t nnz, float* b4,
                        float* diag12, float* val9, const float* ml2, const float* bend_kper,
                        const float* spring_kper)
{
    /* inertia, and the spring / quadratic models when selected; per-element parameters when given */
    orc_material_fill(V, stretch_model == 0 ? E : 0, bending_model == 1 ? B : 0, x4, rest4, xt4, mass, pinned, dt,
                      dirichlet, edges, rest_len, spring_k, spring_kper, stencil, Q16, bending_k, spring_slots,
                      bend_slots, nnz, b4, diag12, val9);
    if (stretch_model == 1) {
        static const int src[6] = {3, 4, 3, 5, 4, 5}, tr[6] = {0, 0, 1, 0, 1, 1};  /* (0,1) (0,2) (1,0) (1,2) (2,0) (2,1) */
#pragma omp parallel for schedule(static)
        for (long long fl = 0; fl < (long long)Fs; ++fl) {
            const size_t f = (size_t)fl;
            const uint32_t* v = sfaces4 + 4 * f;
            float g[9], K[54];
            orc_bw98_face(x4 + 4 * (size_t)v[0], x4 + 4 * (size_t)v[1], x4 + 4 * (size_t)v[2], dm4 + 4 * f,
                          ml2 ? ml2[2 * f] : mu, ml2 ? ml2[2 * f + 1] : lambda, sarea[f], g, K);
            for (int a = 0; a < 3; ++a) {
                for (int k = 0; k < 3; ++k) {
#pragma omp atomic
                    b4[4 * (size_t)v[a] + k] -= g[3 * a + k];
                }
                for (int c = 0; c < 3; ++c)
                    for (int r = 0; r < 3; ++r) {
#pragma omp atomic
                        diag12[12 * (size_t)v[a] + 4 * c + r] += K[9 * a + 3 * c + r];
                    }
            }
            for (int m = 0; m < 6; ++m) {
                float* O = val9 + 9 * (size_t)face_slots[6 * f + m];
                const float* S = K + 9 * src[m];
                for (int c = 0; c < 3; ++c)
                    for (int r = 0; r < 3; ++r) {
#pragma omp atomic
                        O[3 * c + r] += tr[m] ? S[3 * r + c] : S[3 * c + r];
                    }
            }
        }
    }
    if (bending_model == 2) {

#pragma omp parallel for schedule(static)
        for (long long sl = 0; sl < (long long)B; ++sl) {
            const size_t s = (size_t)sl;
            const uint32_t* v = stencil + 4 * s;
            float g[12];
            const float th = orc_dihedral(x4 + 4 * (size_t)v[0], x4 + 4 * (size_t)v[1], x4 + 4 * (size_t)v[2],
                                          x4 + 4 * (size_t)v[3], g);
            const float stiff = ((bend_kper ? bend_kper[s] : bending_k) * bending_scaling) * hbar[s];
            const float sd = stiff * (th - rest_angle[s]);
            int t = 0;
            for (int i = 0; i < 4; ++i) {
                for (int k = 0; k < 3; ++k) {
#pragma omp atomic
                    b4[4 * (size_t)v[i] + k] -= sd * g[3 * i + k];
                }
                for (int j = 0; j < 4; ++j) {
                    float* O = (i == j) ? diag12 + 12 * (size_t)v[i] : val9 + 9 * (size_t)bend_slots[12 * s + t];
                    const int cs = (i == j) ? 4 : 3;  /* diagonal records hold float4 columns */
                    for (int c = 0; c < 3; ++c)
                        for (int r = 0; r < 3; ++r) {
#pragma omp atomic
                            O[cs * c + r] += stiff * (g[3 * i + r] * g[3 * j + c]);
                        }
                    if (i != j) ++t;
                }
            }
        }
    }
}

/*
 * Affine bodies (newton_solver.cpp:1176-1330): per body, b = -grad and the 4 x 4 blocks of inertia
 * (alpha h^-2 M, alpha = 1 + dirichlet for a fixed body) and orthogonality (kappa V sum_ij (a_i.a_j -
 * delta_ij)^2, the reference's gradient and Hessian blocks), written into the DOF slot rows: b and the
 * diagonal stored, off-diagonal blocks (i, j), i != j row-major, at block index body_slots[12 b + t].
 * The operation order follows the CUDA kernel k_abd_body.
 */
void orc_abd_fill(uint32_t NB, const uint32_t* body_dof, const float* mass16, const float* volume, const float* kappa,
                  const uint8_t* fixed, const float* x4, const float* xt4, float dt, float dirichlet,
                  const uint32_t* body_slots, float* b4, float* diag12, float* val9)
{
    const float h2inv = 1.0f / (dt * dt);
    for (uint32_t bi = 0; bi < NB; ++bi) {
        const uint32_t d = body_dof[bi];
        m3 q[4], dq[4];
        for (int j = 0; j < 4; ++j) {
            q[j] = mld(x4, d + j);
            dq[j] = msub(q[j], mld(xt4, d + j));
        }
        const float* M = mass16 + 16 * (size_t)bi;
        const float c = (fixed[bi] ? 1.0f + dirichlet : 1.0f) * h2inv;
        float H[4][4][9];
        m3 G[4];
        for (int i = 0; i < 4; ++i) {
            m3 g = M3(0.0f, 0.0f, 0.0f);
            for (int j = 0; j < 4; ++j) {
                const float m = M[4 * i + j];
                g = M3(g.x + m * dq[j].x, g.y + m * dq[j].y, g.z + m * dq[j].z);
                const float hm = c * m;
                for (int k = 0; k < 9; ++k) H[i][j][k] = (k % 4 == 0) ? hm : 0.0f;
            }
            G[i] = mscl(c, g);
        }
        const float s4 = 4.0f * (kappa[bi] * volume[bi]);
        const m3 A[3] = {q[1], q[2], q[3]};
        for (int ii = 0; ii < 3; ++ii) {
            m3 og = M3(-A[ii].x, -A[ii].y, -A[ii].z);
            for (int jj = 0; jj < 3; ++jj) {
                const float dd = mdot(A[ii], A[jj]);
                og = M3(og.x + dd * A[jj].x, og.y + dd * A[jj].y, og.z + dd * A[jj].z);
            }
            G[1 + ii] = M3(G[1 + ii].x + s4 * og.x, G[1 + ii].y + s4 * og.y, G[1 + ii].z + s4 * og.z);
        }
        for (int ii = 0; ii < 3; ++ii)
            for (int jj = ii; jj < 3; ++jj) {
                const float ai[3] = {A[ii].x, A[ii].y, A[ii].z}, aj[3] = {A[jj].x, A[jj].y, A[jj].z};
                float h[9];
                if (ii == jj) {
                    const float dd = mdot(A[ii], A[ii]) - 1.0f;
                    for (int cc = 0; cc < 3; ++cc)
                        for (int r = 0; r < 3; ++r) {
                            float e = ai[r] * ai[cc] + (r == cc ? dd : 0.0f);
                            for (int k = 0; k < 3; ++k) {
                                const float ak[3] = {A[k].x, A[k].y, A[k].z};
                                e = e + ak[r] * ak[cc];
                            }
                            h[3 * cc + r] = e;
                        }
                } else {
                    const float dd = mdot(A[ii], A[jj]);
                    for (int cc = 0; cc < 3; ++cc)
                        for (int r = 0; r < 3; ++r) h[3 * cc + r] = aj[r] * ai[cc] + (r == cc ? dd : 0.0f);
                }
                for (int cc = 0; cc < 3; ++cc)
                    for (int r = 0; r < 3; ++r) {
                        H[1 + ii][1 + jj][3 * cc + r] = H[1 + ii][1 + jj][3 * cc + r] + s4 * h[3 * cc + r];
                        if (ii != jj)
                            H[1 + jj][1 + ii][3 * r + cc] = H[1 + jj][1 + ii][3 * r + cc] + s4 * h[3 * cc + r];
                    }
            }
        int t = 0;
        for (int i = 0; i < 4; ++i) {
            float* bv = b4 + 4 * (size_t)(d + i);
            bv[0] = -G[i].x;
            bv[1] = -G[i].y;
            bv[2] = -G[i].z;
            bv[3] = 0.0f;
            float* dv = diag12 + 12 * (size_t)(d + i);
            for (int cc = 0; cc < 3; ++cc) {
                for (int r = 0; r < 3; ++r) dv[4 * cc + r] = H[i][i][3 * cc + r];
                dv[4 * cc + 3] = 0.0f;
            }
            for (int j = 0; j < 4; ++j) {
                if (i == j) continue;
                float* O = val9 + 9 * (size_t)body_slots[12 * (size_t)bi + t];
                for (int k = 0; k < 9; ++k) O[k] = H[i][j][k];
                ++t;
            }
        }
    }
}
