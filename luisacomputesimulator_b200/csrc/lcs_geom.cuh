// lcs_geom.cuh -- closest-point coefficients, squared distances, additive CCD and the IPC
// log barrier, as device functions.
//
// Each function follows the device code of the reference (namespace distance:: and accd::;
// the host_* twins differ for EE and are not used):
//   solve / point_edge / point_triangle / edge_edge coeff   Solver/CollisionDetector/distance.hpp:40-110
//   PT unclassified coeff + squared distance              Solver/CollisionDetector/distance.hpp:113-181
//   EE unclassified coeff (with the parallel test)          Solver/CollisionDetector/distance.hpp:245-310
//   centerize / max_relative_u / ccd_helper / PT, EE CCD    Solver/CollisionDetector/accd.hpp:31-205
//   barrier and its two derivatives                        Solver/CollisionDetector/cipc_kernel.hpp:16-36
// The operation order is the oracle's (fma only in dot3), so results match it bit for bit.
#pragma once
#include "lcs_common.cuh"

namespace lcs {

template <typename T>
struct vec3t {
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c);
template <>
__device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <>
__device__ __forceinline__ double fma_t<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T>
struct G {
    using V = vec3t<T>;
    static __device__ __forceinline__ V mk(T x, T y, T z) { return V{x, y, z}; }
    static __device__ __forceinline__ V sub(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
    static __device__ __forceinline__ V add(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
    static __device__ __forceinline__ V scl(T s, V a) { return V{s * a.x, s * a.y, s * a.z}; }
    static __device__ __forceinline__ V neg(V a) { return V{-a.x, -a.y, -a.z}; }
    static __device__ __forceinline__ T dot(V a, V b) { return fma_t<T>(a.z, b.z, fma_t<T>(a.y, b.y, a.x * b.x)); }
    static __device__ __forceinline__ V crs(V a, V b)
    {
        return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    }

    static __device__ __forceinline__ bool solve2(T a00, T a01, T a10, T a11, T b0, T b1, T& x0, T& x1)
    {
        T det = a00 * a11 - a10 * a01;
        if (det != (T)0) {
            T i00 = a11 / det;
            T i01 = -a10 / det;
            T i10 = -a01 / det;
            T i11 = a00 / det;
            x0 = i00 * b0 + i10 * b1;
            x1 = i01 * b0 + i11 * b1;
            return true;
        }
        return false;
    }

    static __device__ __forceinline__ void pe_coeff(V p, V e0, V e1, T& c0, T& c1)
    {
        V r = sub(e1, e0);
        T d = dot(r, r);
        c0 = (T)0.5;
        c1 = (T)0.5;
        if (d > (T)1.19209290E-7f) {
            T x = dot(r, sub(p, e0)) / d;
            c0 = (T)1 - x;
            c1 = x;
        }
    }

    static __device__ __forceinline__ void pt_coeff(V p, V t0, V t1, V t2, T* r)
    {
        V r0 = sub(t1, t0), r1 = sub(t2, t0), w = sub(p, t0);
        T a00 = dot(r0, r0), a01 = dot(r1, r0), a10 = dot(r0, r1), a11 = dot(r1, r1);
        T b0 = dot(r0, w), b1 = dot(r1, w);
        T s0, s1;
        if (!solve2(a00, a01, a10, a11, b0, b1, s0, s1)) {
            s0 = (T)(1.0f / 3.0f);
            s1 = (T)(1.0f / 3.0f);
        }
        T c0 = (T)1 - s0 - s1, c1 = s0, c2 = s1;
        r[0] = c0; r[1] = c1; r[2] = c2;
        if (c0 >= 0 && c1 >= 0 && c2 >= 0 && c0 <= 1 && c1 <= 1 && c2 <= 1) {
        } else if (c0 < 0) {
            T e0, e1;
            pe_coeff(p, t1, t2, e0, e1);
            if (e0 >= 0 && e0 <= 1) { r[0] = 0; r[1] = e0; r[2] = e1; }
            else if (e0 > 1) { r[0] = 0; r[1] = 1; r[2] = 0; }
            else { r[0] = 0; r[1] = 0; r[2] = 1; }
        } else if (c1 < 0) {
            T e0, e1;
            pe_coeff(p, t0, t2, e0, e1);
            if (e0 >= 0 && e0 <= 1) { r[0] = e0; r[1] = 0; r[2] = e1; }
            else if (e0 > 1) { r[0] = 1; r[1] = 0; r[2] = 0; }
            else { r[0] = 0; r[1] = 0; r[2] = 1; }
        } else {
            T e0, e1;
            pe_coeff(p, t0, t1, e0, e1);
            if (e0 >= 0 && e0 <= 1) { r[0] = e0; r[1] = e1; r[2] = 0; }
            else if (e0 > 1) { r[0] = 1; r[1] = 0; r[2] = 0; }
            else { r[0] = 0; r[1] = 1; r[2] = 0; }
        }
    }

    static __device__ __forceinline__ T pt_dist2(V p, V t0, V t1, V t2)
    {
        T c[3];
        pt_coeff(p, t0, t1, t2, c);
        V x = add(add(scl(c[0], sub(t0, p)), scl(c[1], sub(t1, p))), scl(c[2], sub(t2, p)));
        return dot(x, x);
    }

    static __device__ __forceinline__ T clamp01(T v)
    {
        T lo = v > (T)0 ? v : (T)0;
        return lo < (T)1 ? lo : (T)1;
    }

    static __device__ __forceinline__ void ee_coeff(V ea0, V ea1, V eb0, V eb1, T* res)
    {
        V r0 = sub(ea1, ea0), r1 = sub(eb1, eb0);
        T len0 = dot(r0, r0), len1 = dot(r1, r1);
        V cr = crs(r0, r1);
        T pm = dot(cr, cr) / (len0 * len1 + (T)1e-8f);
        V m1 = neg(r1), w = sub(eb0, ea0);
        T a00 = dot(r0, r0), a01 = dot(m1, r0), a10 = dot(r0, m1), a11 = dot(m1, m1);
        T b0 = dot(r0, w), b1 = dot(m1, w);
        T c0 = (T)0.5, c1 = (T)0.5, c2 = (T)0.5, c3 = (T)0.5;
        T s0, s1;
        if (solve2(a00, a01, a10, a11, b0, b1, s0, s1)) {
            c0 = (T)1 - s0; c1 = s0; c2 = (T)1 - s1; c3 = s1;
        }
        res[0] = c0; res[1] = c1; res[2] = c2; res[3] = c3;
        bool valid = c0 >= 0 && c1 >= 0 && c2 >= 0 && c3 >= 0 && c0 <= 1 && c1 <= 1 && c2 <= 1 && c3 <= 1;
        if (pm < (T)1e-4f || !valid) {
            T k[4][4];
            T a, b;
            pe_coeff(ea0, eb0, eb1, a, b);
            k[0][0] = 1; k[0][1] = 0; k[0][2] = clamp01(a); k[0][3] = clamp01(b);
            pe_coeff(ea1, eb0, eb1, a, b);
            k[1][0] = 0; k[1][1] = 1; k[1][2] = clamp01(a); k[1][3] = clamp01(b);
            pe_coeff(eb0, ea0, ea1, a, b);
            k[2][0] = clamp01(a); k[2][1] = clamp01(b); k[2][2] = 1; k[2][3] = 0;
            pe_coeff(eb1, ea0, ea1, a, b);
            k[3][0] = clamp01(a); k[3][1] = clamp01(b); k[3][2] = 0; k[3][3] = 1;
            int index = 0;
            T min_d = (T)3.402823466e+38F;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                V x0 = add(scl(k[i][0], ea0), scl(k[i][1], ea1));
                V x1 = add(scl(k[i][2], eb0), scl(k[i][3], eb1));
                V dd = sub(x0, x1);
                T d = dot(dd, dd);
                if (d < min_d) { min_d = d; index = i; }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (i == index) { res[0] = k[i][0]; res[1] = k[i][1]; res[2] = k[i][2]; res[3] = k[i][3]; }
        }
    }

    static __device__ __forceinline__ T ee_dist2(V ea0, V ea1, V eb0, V eb1)
    {
        T c[4];
        ee_coeff(ea0, ea1, eb0, eb1, c);
        V x0 = add(scl(c[0], ea0), scl(c[1], ea1));
        V x1 = add(scl(c[2], eb0), scl(c[3], eb1));
        V dd = sub(x1, x0);
        return dot(dd, dd);
    }

    template <bool EE>
    static __device__ __forceinline__ T dist2(const V* x)
    {
        if (EE) return ee_dist2(x[0], x[1], x[2], x[3]);
        return pt_dist2(x[0], x[1], x[2], x[3]);
    }
};

using Gf = G<float>;
using Gd = G<double>;
using vf = vec3t<float>;
using vd = vec3t<double>;

__device__ __forceinline__ vf tovf(v3 a) { return vf{a.x, a.y, a.z}; }

// accd.hpp:49-101, with the precision form's FP64 re-check of the final iterate (flag)
template <bool EE>
__device__ __forceinline__ float ccd_helper(const vf* x0, const vf* dx, float u_max, float offset, bool fp64_final)
{
    float toi = 0.0f, prev = 0.0f;
    const float max_t = 1.25f;
    float eps = 0.01f * (sqrtf(Gf::dist2<EE>(x0)) - offset);
    float target = eps + offset;
    float eps_sqr = eps * eps;
    float inv_u_max = 1.0f / u_max;
    unsigned iter = 0;
    bool contact = false;
    for (;;) {
        if (iter > 10000u) { toi = 0.001f; break; }
        iter++;
        vf xt[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) xt[k] = Gf::add(x0[k], Gf::scl(toi, dx[k]));
        float d2 = Gf::dist2<EE>(xt);
        float dmt = (d2 - target * target) / (sqrtf(d2) + target);
        if ((max_t - toi) * u_max < dmt - eps) { toi = max_t; break; }
        else if (toi > 0.0f && dmt * dmt < eps_sqr) { contact = true; break; }
        float toi_next = toi + dmt * inv_u_max;
        if (toi_next != toi) { prev = toi; toi = toi_next; }
        else { contact = true; break; }
        if (toi > max_t) { toi = max_t; break; }
    }
    if (fp64_final && contact && toi > 0.0f) {
        vd xd[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            xd[k] = Gd::add(vd{x0[k].x, x0[k].y, x0[k].z}, Gd::scl((double)toi, vd{dx[k].x, dx[k].y, dx[k].z}));
        double d = sqrt(Gd::dist2<EE>(xd));
        if (!(d > (double)offset)) toi = prev;
        toi = nextafterf(toi, 0.0f);
    }
    return toi;
}

__device__ __forceinline__ void centerize(vf* x)
{
    vf mov = vf{0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 4; ++k) mov = Gf::add(mov, Gf::scl(0.25f, x[k]));
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = Gf::sub(x[k], mov);
}

__device__ __forceinline__ float max_relative_u(const vf* u)
{
    float m = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i + 1; j < 4; ++j) {
            vf du = Gf::sub(u[i], u[j]);
            m = fmx(m, Gf::dot(du, du));
        }
    return sqrtf(m);
}

// accd.hpp:143-171 (EE = false) and 173-202 (EE = true); a = begin positions, b = end positions
template <bool EE>
__device__ __forceinline__ float accd_ccd(const v3* a, const v3* b, float offset, bool fp64_final)
{
    vf x0[4], dx[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        x0[k] = tovf(a[k]);
        dx[k] = Gf::sub(tovf(b[k]), tovf(a[k]));
    }
    centerize(x0);
    centerize(dx);
    float u_max = max_relative_u(dx);
    float toi = 1.25f;
    if (u_max != 0.0f) toi = ccd_helper<EE>(x0, dx, u_max, offset, fp64_final);
    return toi;
}

// The same additive CCD carried out entirely in double precision (positions promoted exactly,
// offset promoted): the precision form's step bound.  Returns the FP64 time of impact; the
// caller rounds it toward zero so the float it stores never exceeds it.
template <bool EE>
__device__ __forceinline__ double accd_ccd_f64(const v3* a, const v3* b, float offset_f)
{
    vd x0[4], dx[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        x0[k] = vd{a[k].x, a[k].y, a[k].z};
        dx[k] = Gd::sub(vd{b[k].x, b[k].y, b[k].z}, x0[k]);
    }
    vd m0 = vd{0.0, 0.0, 0.0}, m1 = vd{0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        m0 = Gd::add(m0, Gd::scl(0.25, x0[k]));
        m1 = Gd::add(m1, Gd::scl(0.25, dx[k]));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        x0[k] = Gd::sub(x0[k], m0);
        dx[k] = Gd::sub(dx[k], m1);
    }
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i + 1; j < 4; ++j) {
            const vd du = Gd::sub(dx[i], dx[j]);
            const double q = Gd::dot(du, du);
            m = q > m ? q : m;
        }
    const double u_max = sqrt(m);
    const double max_t = 1.25;
    if (u_max == 0.0) return max_t;
    const double offset = offset_f;
    double toi = 0.0;
    const double eps = 0.01 * (sqrt(Gd::dist2<EE>(x0)) - offset);
    const double target = eps + offset, eps_sqr = eps * eps, inv_u_max = 1.0 / u_max;
    for (unsigned iter = 0;; ++iter) {
        if (iter > 10000u) return 0.001;
        vd xt[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) xt[k] = Gd::add(x0[k], Gd::scl(toi, dx[k]));
        const double d2 = Gd::dist2<EE>(xt);
        const double dmt = (d2 - target * target) / (sqrt(d2) + target);
        if ((max_t - toi) * u_max < dmt - eps) return max_t;
        if (toi > 0.0 && dmt * dmt < eps_sqr) break;
        const double nt = toi + dmt * inv_u_max;
        if (nt == toi) break;
        toi = nt;
        if (toi > max_t) return max_t;
    }
    return toi;
}

// cipc_kernel.hpp:16-36
__device__ __forceinline__ float barrier_e(float d, float dhat)
{
    float t = d - dhat;
    return -t * t * logf(d / dhat);
}
__device__ __forceinline__ float barrier_d1(float d, float dhat)
{
    return (dhat - d) * (2.0f * logf(d / dhat) - dhat / d + 1.0f);
}
__device__ __forceinline__ float barrier_d2(float d, float dhat)
{
    float q = dhat / d;
    return (q + 2.0f) * q - 2.0f * logf(d / dhat) - 3.0f;
}

// pairs of a list whose count lives on the device: min(count, capacity)
__device__ __forceinline__ uint32_t pair_count(const uint32_t* d_count, uint32_t cap)
{
    uint32_t n = *d_count;
    return n < cap ? n : cap;
}

struct PairView {
    uint32_t v[4];
    float w[4];
    v3 n;
    float k1, k2, stiff;
    int type;  // 0 none, 1 VF, 2 EE
};

// CollisionPairTemplate::get_weight, collision_data.h:308-324
__device__ __forceinline__ PairView load_pair(const lcs_pair* pairs, uint32_t k)
{
    const uint4* r = reinterpret_cast<const uint4*>(pairs + k);
    const uint4 id = __ldg(r);
    const float4 a = __ldg(reinterpret_cast<const float4*>(r) + 1);
    const float4 b = __ldg(reinterpret_cast<const float4*>(r) + 2);
    PairView P;
    P.v[0] = id.x & 0x7FFFFFFFu; P.v[1] = id.y & 0x7FFFFFFFu; P.v[2] = id.z & 0x7FFFFFFFu; P.v[3] = id.w & 0x7FFFFFFFu;
    P.n = mk3(a.x, a.y, a.z);
    P.stiff = a.w;
    P.k1 = b.x;
    P.k2 = b.y;
    if (id.z >> 31) {
        P.type = 1;
        P.w[0] = 1.0f; P.w[1] = -b.z; P.w[2] = -b.w; P.w[3] = b.z + b.w - 1.0f;
    } else if (id.w >> 31) {
        P.type = 2;
        P.w[0] = b.z; P.w[1] = 1.0f - b.z; P.w[2] = -b.w; P.w[3] = b.w - 1.0f;
    } else {
        P.type = 0;
        P.w[0] = P.w[1] = P.w[2] = P.w[3] = 0.0f;
    }
    return P;
}


}  // namespace lcs
