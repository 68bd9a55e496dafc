// lbvh_common.cuh -- device helpers shared by the single-tree LBVH (lbvh.cu) and the forest of
// per-scene trees used by the batched solver (forest.cu): Morton codes, element boxes, the Karras
// common-prefix helper, leaf boxes and the 64-B traversal records.
#pragma once
#include "lcs_common.cuh"
#include "../../include/lcs_gpu.h"

namespace lcs {

__device__ __forceinline__ uint32_t expand_bits(uint32_t v)
{
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    return (v | (v << 2)) & 0x09249249u;
}

// make_morton32, lbvh.cpp:112-124
__device__ __forceinline__ uint32_t morton32(float px, float py, float pz)
{
    float x = fmn(fmx(px * 1024.0f, 0.0f), 1023.0f);
    float y = fmn(fmx(py * 1024.0f, 0.0f), 1023.0f);
    float z = fmn(fmx(pz * 1024.0f, 0.0f), 1023.0f);
    return (expand_bits((uint32_t)x) << 2) | (expand_bits((uint32_t)y) << 1) | expand_bits((uint32_t)z);
}

__device__ __forceinline__ void elem_box(int kind, const float4* __restrict__ x, const uint32_t* __restrict__ elems,
                                         uint32_t e, v3& mn, v3& mx, v3& c)
{
    if (kind == LCS_TREE_VERT) {
        v3 p = ld3(x, e);
        mn = p; mx = p; c = p;
    } else if (kind == LCS_TREE_EDGE) {
        uint2 ed = __ldg(reinterpret_cast<const uint2*>(elems) + e);
        v3 p0 = ld3(x, ed.x), p1 = ld3(x, ed.y);
        mn = min3(p0, p1);
        mx = max3(p0, p1);
        c = 0.5f * (p0 + p1);  // lbvh.cpp:468
    } else {
        uint4 f = __ldg(reinterpret_cast<const uint4*>(elems) + e);
        v3 p0 = ld3(x, f.x), p1 = ld3(x, f.y), p2 = ld3(x, f.z);
        mn = min3(p0, min3(p1, p2));
        mx = max3(p0, max3(p1, p2));
        c = 0.333333f * ((p0 + p1) + p2);  // lbvh.cpp:488
    }
}

__device__ __forceinline__ int cp_ij(uint64_t mi, int j, const uint64_t* __restrict__ ms, int n)
{
    return (j >= 0 && j < n) ? __clzll((long long)(mi ^ ms[j])) : -1;
}

__device__ __forceinline__ void leaf_box(int kind, uint32_t e, const float* __restrict__ thickness,
                                         const float4* __restrict__ x0, const float4* __restrict__ x1,
                                         const uint32_t* __restrict__ elems, v3& mn, v3& mx)
{
    float th;
    if (kind == LCS_TREE_VERT) {
        v3 a = ld3(x0, e), b = ld3(x1, e);
        mn = min3(a, b);
        mx = max3(a, b);
        th = __ldg(&thickness[e]);
    } else if (kind == LCS_TREE_EDGE) {
        uint2 ed = __ldg(reinterpret_cast<const uint2*>(elems) + e);
        v3 s0 = ld3(x0, ed.x), s1 = ld3(x0, ed.y), e0 = ld3(x1, ed.x), e1 = ld3(x1, ed.y);
        mn = min3(min3(s0, s1), min3(e0, e1));
        mx = max3(max3(s0, s1), max3(e0, e1));
        th = __ldg(&thickness[ed.x]);
    } else {
        uint4 f = __ldg(reinterpret_cast<const uint4*>(elems) + e);
        v3 s0 = ld3(x0, f.x), s1 = ld3(x0, f.y), s2 = ld3(x0, f.z);
        v3 e0 = ld3(x1, f.x), e1 = ld3(x1, f.y), e2 = ld3(x1, f.z);
        mn = min3(min3(s0, min3(s1, s2)), min3(e0, min3(e1, e2)));
        mx = max3(max3(s0, max3(s1, s2)), max3(e0, max3(e1, e2)));
        th = __ldg(&thickness[f.x]);
    }
    mn = mk3(mn.x - th, mn.y - th, mn.z - th);
    mx = mk3(mx.x + th, mx.y + th, mx.z + th);
}

// slot s of the node records: {min.xyz | code}{max.xyz | last}, `last` being the largest sorted leaf
// position under the slot (the pruning key of the once-per-pair EE traversal)
__device__ __forceinline__ void store_slot(float4* wide, uint32_t s, v3 mn, v3 mx, uint32_t code, uint32_t last = 0u)
{
    float4* r = wide + 4 * (s >> 1) + 2 * (s & 1u);
    __stcg(r, make_float4(mn.x, mn.y, mn.z, __uint_as_float(code)));
    __stcg(r + 1, make_float4(mx.x, mx.y, mx.z, __uint_as_float(last)));
}

// one record slot {min.xyz | code}{max.xyz | last} as a single 32-byte read-only load (slots are 32-byte
// aligned): a lane's walk step then costs the L1 half the requests of two 16-byte loads
__device__ __forceinline__ void ld_slot(const float4* p, float4& mn, float4& mx)
{
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(mn.x), "=f"(mn.y), "=f"(mn.z), "=f"(mn.w), "=f"(mx.x), "=f"(mx.y), "=f"(mx.z), "=f"(mx.w)
        : "l"(p));
}

// the strict overlap test of AABB::is_overlap_aabb (aabb.h:95-100); q = {min xyz, max xyz}
__device__ __forceinline__ bool overlap(float4 mn, float4 mx, const float* q)
{
    return mn.x < q[3] && mn.y < q[4] && mn.z < q[5] && mx.x > q[0] && mx.y > q[1] && mx.z > q[2];
}

}  // namespace lcs
