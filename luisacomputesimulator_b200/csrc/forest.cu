// forest.cu -- a forest of per-scene LBVHs held in one set of device arrays, for the batched
// solver (many independent scenes stepped by the same launches).
//
// Every scene's tree is the tree lcs_bvh builds for that scene alone (LBVH::construct_tree,
// Solver/CollisionDetector/lbvh.cpp:939-998): the scene's own global AABB with the reference's
// ceil(n_verts / 256)-block cover (lbvh.cpp:958, 968), its own Morton normalisation
// (lbvh.cpp:507-523), a stable sort of its elements by Morton code, and Karras inner nodes over
// morton64 = code << 32 | LOCAL element index (lbvh.cpp:155-291, 541-596), so that its topology,
// refit boxes and query results are bit-identical to the standalone tree.  One launch covers all
// scenes: the sort key is scene << 30 | code (one 64-bit LSD radix sort keeps every scene's
// elements contiguous and in their standalone order), each inner node and leaf knows its scene,
// and a query starts at the root of its own scene.
//
// Global node ids: inner nodes of scene s are [ioff[s], ioff[s] + n_s - 1) (root ioff[s]); the
// leaf at sorted position i (global) is NI + i.  Traversal records (`wide`, one 64-B record per
// inner node) and child codes are as in lbvh.cu: inner child -> global inner id, leaf child ->
// 0x80000000 | global element id.  Scenes must have at least two elements.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "lbvh_common.cuh"
#include "lcs_common.cuh"
#include "lcs_internal.h"
#include "radix_sort.cuh"

using namespace lcs;

struct lcs_forest {
    int kind = 0;
    uint32_t S = 0, N = 0, NI = 0, NB = 0, sbits = 0;
    std::vector<uint32_t> h_eoff, h_ioff;
    uint32_t *eoff = nullptr, *ioff = nullptr, *boff = nullptr, *bcover = nullptr;
    uint32_t *escene = nullptr, *iscene = nullptr, *bscene = nullptr;
    float4* centers = nullptr;
    float* block_aabb = nullptr;
    float* gaabb = nullptr;
    uint32_t* m30 = nullptr;
    uint64_t *keys = nullptr, *keys_alt = nullptr;
    uint32_t *vals = nullptr, *vals_alt = nullptr, *hist = nullptr;
    uint32_t* sgo = nullptr;      // points into vals or vals_alt
    uint64_t* skeys = nullptr;    // sorted keys (points into keys or keys_alt)
    uint64_t* ms64 = nullptr;
    uint32_t* parent = nullptr;   // NI + N
    uint2* children = nullptr;    // NI + N
    uint32_t* slot = nullptr;     // NI + N
    float4* wide = nullptr;       // 4 NI
    uint32_t* counters = nullptr; // NI
    uint32_t* healthy = nullptr;
    uint32_t* saved_count = nullptr;  // 1: the candidate count before a tuning query (restored between trials)
    bool built = false;               // a build has written the sorted order, topology and slots
    mutable uint32_t q_threads = 0;   // tuned threads per block of the queries (0: not tuned yet)
    mutable float q_ms = 0.0f;        // the tuned configuration's query time
};

namespace {

// fn_reduce_{edge,face}_tree_global_aabb per scene: centres + per-256-element block partials
__global__ void __launch_bounds__(256) k_f_pass1(int kind, const float4* __restrict__ x,
                                                 const uint32_t* __restrict__ elems, const uint32_t* __restrict__ eoff,
                                                 const uint32_t* __restrict__ boff, const uint32_t* __restrict__ bscene,
                                                 float4* __restrict__ centers, float* __restrict__ block_aabb)
{
    __shared__ float red[8][6];
    const uint32_t s = bscene[blockIdx.x];
    const uint32_t e = eoff[s] + (blockIdx.x - boff[s]) * 256 + threadIdx.x;
    v3 mn = mk3(INFINITY, INFINITY, INFINITY), mx = mk3(-INFINITY, -INFINITY, -INFINITY);
    if (e < eoff[s + 1]) {
        v3 c;
        elem_box(kind, x, elems, e, mn, mx, c);
        centers[e] = make_float4(c.x, c.y, c.z, 0.0f);
    }
    float v[6] = {mn.x, mn.y, mn.z, mx.x, mx.y, mx.z};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float t = __shfl_xor_sync(0xFFFFFFFFu, v[k], o);
            v[k] = k < 3 ? fmn(v[k], t) : fmx(v[k], t);
        }
    if (lane_id() == 0)
#pragma unroll
        for (int k = 0; k < 6; ++k) red[threadIdx.x >> 5][k] = v[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        float r = red[0][threadIdx.x];
        for (int w = 1; w < 8; ++w) r = threadIdx.x < 3 ? fmn(r, red[w][threadIdx.x]) : fmx(r, red[w][threadIdx.x]);
        block_aabb[6 * blockIdx.x + threadIdx.x] = r;
    }
}

// fn_reduce_aabb_2_pass per scene (one block per scene) over the scene's first bcover partials
__global__ void __launch_bounds__(256) k_f_pass2(const float* __restrict__ block_aabb, const uint32_t* __restrict__ boff,
                                                 const uint32_t* __restrict__ bcover, float* __restrict__ gaabb)
{
    __shared__ float red[8][6];
    const uint32_t s = blockIdx.x, b0 = boff[s], nb = bcover[s];
    float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (uint32_t b = threadIdx.x; b < nb; b += 256)
#pragma unroll
        for (int k = 0; k < 6; ++k)
            v[k] = k < 3 ? fmn(v[k], block_aabb[6 * (b0 + b) + k]) : fmx(v[k], block_aabb[6 * (b0 + b) + k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float t = __shfl_xor_sync(0xFFFFFFFFu, v[k], o);
            v[k] = k < 3 ? fmn(v[k], t) : fmx(v[k], t);
        }
    if (lane_id() == 0)
#pragma unroll
        for (int k = 0; k < 6; ++k) red[threadIdx.x >> 5][k] = v[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        float r = red[0][threadIdx.x];
        for (int w = 1; w < 8; ++w) r = threadIdx.x < 3 ? fmn(r, red[w][threadIdx.x]) : fmx(r, red[w][threadIdx.x]);
        gaabb[6 * s + threadIdx.x] = r;
    }
}

// fn_compute_mortons with the element's own scene box; sort key = scene << 30 | code
__global__ void k_f_mortons(const float4* __restrict__ centers, const float* __restrict__ gaabb,
                            const uint32_t* __restrict__ escene, uint32_t n, uint32_t* __restrict__ m30,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = escene[i];
        const float* g = gaabb + 6 * s;
        const float inv0 = 1.0f / fmx(g[3] - g[0], 1e-6f);
        const float inv1 = 1.0f / fmx(g[4] - g[1], 1e-6f);
        const float inv2 = 1.0f / fmx(g[5] - g[2], 1e-6f);
        const float4 c = centers[i];
        const uint32_t m = morton32((c.x - g[0]) * inv0, (c.y - g[1]) * inv1, (c.z - g[2]) * inv2);
        m30[i] = m;
        keys[i] = ((uint64_t)s << 30) | m;
        vals[i] = i;
    }
}

// fn_reset_tree + fn_apply_sorted per scene: morton64 over the LOCAL element index
__global__ void k_f_apply(const uint64_t* __restrict__ skeys, const uint32_t* __restrict__ sgo,
                          const uint32_t* __restrict__ escene, const uint32_t* __restrict__ eoff,
                          const uint32_t* __restrict__ ioff, uint32_t n, uint32_t NI, uint64_t* __restrict__ ms64,
                          uint2* __restrict__ children, uint32_t* __restrict__ parent, uint32_t* __restrict__ healthy)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = escene[i];  // sorted positions of scene s are [eoff[s], eoff[s+1])
        const uint32_t e = sgo[i];
        ms64[i] = ((skeys[i] & 0x3FFFFFFFull) << 32) | (uint64_t)(e - eoff[s]);
        children[NI + i] = make_uint2(e, e);
        if (i == eoff[s]) parent[ioff[s]] = kInvalid;
        if (i == 0) *healthy = 1u;
    }
}

// fn_build_inner_nodes per scene (local Karras over the scene's sorted segment), global ids out
__global__ void k_f_build_inner(const uint64_t* __restrict__ ms_all, const uint32_t* __restrict__ sgo,
                                const uint32_t* __restrict__ iscene, const uint32_t* __restrict__ eoff,
                                const uint32_t* __restrict__ ioff, uint32_t NI, uint32_t* __restrict__ parent,
                                uint2* __restrict__ children, uint32_t* __restrict__ slot, float4* __restrict__ wide)
{
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < NI; g += gridDim.x * blockDim.x) {
        const uint32_t s = iscene[g];
        const uint32_t e0 = eoff[s], io = ioff[s];
        const int n = (int)(eoff[s + 1] - e0), ni = n - 1;
        const uint64_t* ms = ms_all + e0;
        const int nid = (int)(g - io);
        int i = 0, j = ni;
        if (nid != 0) {
            const uint64_t mi = ms[nid];
            const int cl = __clzll((long long)(mi ^ ms[nid - 1]));
            const int cr = __clzll((long long)(mi ^ ms[nid + 1]));
            const int d = cl < cr ? 1 : -1;
            const int cp_min = cl < cr ? cl : cr;
            int lmax = 2;
            while (cp_ij(mi, nid + lmax * d, ms, n) > cp_min) lmax <<= 1;
            int l = 0;
            for (int t = lmax >> 1; t >= 1; t >>= 1)
                if (cp_ij(mi, nid + (l + t) * d, ms, n) > cp_min) l += t;
            i = nid;
            j = nid + l * d;
        }
        const int a = i < j ? i : j, b = i < j ? j : i;
        int split;
        {
            const uint64_t ma = ms[a], mb = ms[b];
            if (ma == mb) {
                split = (a + b) >> 1;
            } else {
                const int cp_node = __clzll((long long)(ma ^ mb));
                int t = b - a;
                split = a;
                for (;;) {
                    t = (t + 1) >> 1;
                    const int ns = split + t;
                    if (ns < b && __clzll((long long)(ma ^ ms[ns])) > cp_node) split = ns;
                    if (!(t > 1)) break;
                }
            }
        }
        int cleft = (a == split) ? ni + split : split;
        int cright = (b == split + 1) ? ni + split + 1 : split + 1;
        if (cright >= ni) {
            const int t = cleft;
            cleft = cright;
            cright = t;
        }
        // local -> global: inner c -> io + c; leaf ni + p -> NI + e0 + p
        const uint32_t gl = cleft < ni ? io + (uint32_t)cleft : NI + e0 + (uint32_t)(cleft - ni);
        const uint32_t gr = cright < ni ? io + (uint32_t)cright : NI + e0 + (uint32_t)(cright - ni);
        parent[gl] = g;
        parent[gr] = g;
        children[g] = make_uint2(gl, gr);
        slot[gl] = 2u * g + 0u;
        slot[gr] = 2u * g + 1u;
        const uint32_t code_l = cleft < ni ? gl : (0x80000000u | sgo[e0 + (uint32_t)(cleft - ni)]);
        const uint32_t code_r = cright < ni ? gr : (0x80000000u | sgo[e0 + (uint32_t)(cright - ni)]);
        wide[4 * g + 0].w = __uint_as_float(code_l);
        wide[4 * g + 2].w = __uint_as_float(code_r);
    }
}

__global__ void k_f_check(const uint2* __restrict__ children, const uint32_t* __restrict__ parent, uint32_t NI,
                          uint32_t* __restrict__ healthy)
{
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < NI; g += gridDim.x * blockDim.x) {
        const uint2 c = children[g];
        if (parent[c.x] != g || parent[c.y] != g) *healthy = 0u;
    }
}

__device__ __forceinline__ unsigned atom_add_acq_rel_f(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// leaf update + the reference's bottom-up refit walk (fn_refit_tree_aabb, lbvh.cpp:702-754): the second child to
// arrive at a node unions the two boxes and goes on up; a scene's root has no parent
__global__ void k_f_refit(int kind, uint32_t n, uint32_t NI, const uint32_t* __restrict__ sgo,
                          const uint32_t* __restrict__ slot, const uint32_t* __restrict__ parent,
                          const float* __restrict__ thickness, const float4* __restrict__ x0,
                          const float4* __restrict__ x1, const uint32_t* __restrict__ elems, float4* wide,
                          uint32_t* counters, uint32_t* healthy)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = sgo[i];
        v3 mn, mx;
        leaf_box(kind, e, thickness, x0, x1, elems, mn, mx);
        store_slot(wide, slot[NI + i], mn, mx, 0x80000000u | e);
        uint32_t p = parent[NI + i];
        for (int guard = 0;; ++guard) {
            if (guard > 256 || p >= NI) {
                *healthy = 0u;
                break;
            }
            if (atom_add_acq_rel_f(&counters[p], 1u) == 0u) break;  // first arrival: the sibling finishes
            counters[p] = 0u;
            const float4* r = wide + 4 * p;
            const float4 a0 = __ldcg(r + 0), a1 = __ldcg(r + 1), b0 = __ldcg(r + 2), b1 = __ldcg(r + 3);
            const uint32_t pp = parent[p];
            if (pp == kInvalid) break;  // the scene's root: its box is not stored anywhere
            const v3 bmn = mk3(fmn(a0.x, b0.x), fmn(a0.y, b0.y), fmn(a0.z, b0.z));
            const v3 bmx = mk3(fmx(a1.x, b1.x), fmx(a1.y, b1.y), fmx(a1.z, b1.z));
            store_slot(wide, slot[p], bmn, bmx, p);
            p = pp;
        }
    }
}

// query_template2 from the root of the query's own scene (fn_query_from_verts_v2 / _edges_v2)
template <bool EE>
__global__ void __launch_bounds__(256) k_f_query(const float4* __restrict__ wide, const uint32_t* __restrict__ ioff,
                                                 const uint32_t* __restrict__ qscene, const float4* __restrict__ x0,
                                                 const float4* __restrict__ x1, const uint2* __restrict__ edges,
                                                 uint32_t n_queries, const float* __restrict__ dhat,
                                                 const float* __restrict__ thickness, uint2* __restrict__ pairs,
                                                 uint32_t capacity, uint32_t* d_count, const uint32_t* __restrict__ order,
                                                 uint32_t* capped, const uint8_t* __restrict__ only)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_queries; t += gridDim.x * blockDim.x) {
        const uint32_t q = order ? __ldg(&order[t]) : t;
        if (only && !only[EE ? __ldg(&edges[q]).x : q]) continue;  // queries of the masked scenes only
        float box[6];
        {
            v3 mn, mx;
            uint32_t v0;
            if (EE) {
                const uint2 ed = __ldg(&edges[q]);
                const v3 s0 = ld3(x0, ed.x), s1 = ld3(x0, ed.y), e0 = ld3(x1, ed.x), e1 = ld3(x1, ed.y);
                mn = min3(min3(s0, s1), min3(e0, e1));
                mx = max3(max3(s0, s1), max3(e0, e1));
                v0 = ed.x;
            } else {
                const v3 a = ld3(x0, q), b = ld3(x1, q);
                mn = min3(a, b);
                mx = max3(a, b);
                v0 = q;
            }
            const float dh = __ldg(&dhat[v0]);
            const float r = __ldg(&thickness[v0]) + dh;
            box[0] = mn.x - r; box[1] = mn.y - r; box[2] = mn.z - r;
            box[3] = mx.x + r; box[4] = mx.y + r; box[5] = mx.z + r;
            if (!EE && dh < 0.0f) {  // a vertex with a negative d_hat (affine-body DOF slot) queries nothing
                box[0] = box[1] = box[2] = __int_as_float(0x7f800000);
                box[3] = box[4] = box[5] = __int_as_float(0xff800000);
            }
        }
        uint32_t stack[32];
        int sp = 0;
        uint32_t loop = 0;
        stack[sp++] = __ldg(&ioff[__ldg(&qscene[q])]);
        while (sp > 0) {
            const uint32_t node = stack[--sp];
            const float4* r = wide + 4 * node;
            float4 a0, a1, b0, b1;
            ld_slot(r, a0, a1);
            ld_slot(r + 2, b0, b1);
            bool stop = false;
            uint32_t hit[2];
            uint32_t nhit = 0;
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const float4 mn = side ? b0 : a0, mx = side ? b1 : a1;
                if (!stop && overlap(mn, mx, box)) {
                    const uint32_t code = __float_as_uint(mn.w);
                    if (code & 0x80000000u) {
                        const uint32_t obj = code & 0x7FFFFFFFu;
                        if (!EE || q < obj) hit[nhit++] = obj;
                    } else if (sp < 32) {
                        stack[sp++] = code;
                    } else {
                        stop = true;  // a full stack ends the whole traversal (lbvh.cpp:344-351)
                    }
                }
            }
            const uint32_t active = __activemask();
            const uint32_t lt = (1u << lane_id()) - 1u;
            const uint32_t one = __ballot_sync(active, nhit >= 1), two = __ballot_sync(active, nhit == 2);
            const uint32_t total = __popc(one) + __popc(two);
            const uint32_t leader = __ffs(active) - 1;
            uint32_t base = 0;
            if (lane_id() == leader && total) base = atomicAdd(d_count, total);
            base = __shfl_sync(active, base, leader) + __popc(one & lt) + __popc(two & lt);
            for (uint32_t k = 0; k < nhit; ++k)
                if (base + k < capacity) pairs[base + k] = make_uint2(q, hit[k]);
            if (stop || ++loop > 100000u) {
                if (capped) atomicOr(capped, 1u);
                break;
            }
        }
    }
}

struct ForestView {  // the device arrays k_f_export reads (kernel parameters must be plain data)
    const uint32_t *eoff, *ioff, *parent, *slot, *sgo;
    const uint2* children;
    const uint64_t* ms64;
    const float4* wide;
    uint32_t NI;
};

// one scene's tree in the standalone LbvhData layout (local ids), for tests and interop
__global__ void k_f_export(const ForestView f, uint32_t s, uint32_t* __restrict__ parent, uint2* __restrict__ children,
                           uint32_t* __restrict__ object_idx, uint64_t* __restrict__ morton_sorted,
                           uint32_t* __restrict__ sgo_out, float* __restrict__ node_aabb)
{
    const uint32_t e0 = f.eoff[s], n = f.eoff[s + 1] - e0, ni = n - 1, io = f.ioff[s];
    auto to_local = [&](uint32_t g) -> uint32_t {
        if (g == kInvalid) return kInvalid;
        return g < f.NI ? g - io : ni + (g - f.NI - e0);
    };
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < 2 * n - 1; k += gridDim.x * blockDim.x) {
        const uint32_t g = k < ni ? io + k : f.NI + e0 + (k - ni);
        if (parent) parent[k] = to_local(f.parent[g]);
        if (children) {
            const uint2 c = f.children[g];
            children[k] = k < ni ? make_uint2(to_local(c.x), to_local(c.y)) : make_uint2(c.x - e0, c.y - e0);
        }
        if (object_idx) object_idx[k] = k >= ni ? f.sgo[e0 + k - ni] - e0 : kInvalid;
        if (k < n) {
            if (morton_sorted) morton_sorted[k] = f.ms64[e0 + k];
            if (sgo_out) sgo_out[k] = f.sgo[e0 + k] - e0;
        }
        if (node_aabb) {
            float4 mn, mx;
            if (k == 0) {
                const float4 a0 = f.wide[4 * io], a1 = f.wide[4 * io + 1], b0 = f.wide[4 * io + 2], b1 = f.wide[4 * io + 3];
                mn = make_float4(fmn(a0.x, b0.x), fmn(a0.y, b0.y), fmn(a0.z, b0.z), 0.0f);
                mx = make_float4(fmx(a1.x, b1.x), fmx(a1.y, b1.y), fmx(a1.z, b1.z), 0.0f);
            } else {
                const uint32_t sl = f.slot[g];
                mn = f.wide[4 * (sl >> 1) + 2 * (sl & 1u)];
                mx = f.wide[4 * (sl >> 1) + 2 * (sl & 1u) + 1];
            }
            float* o = node_aabb + 8 * (size_t)k;
            o[0] = mn.x; o[1] = mn.y; o[2] = mn.z; o[3] = 0.0f;
            o[4] = mx.x; o[5] = mx.y; o[6] = mx.z; o[7] = 0.0f;
        }
    }
}

template <typename T>
cudaError_t dalloc(T*& p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (count ? count : 1));
}

template <typename T>
cudaError_t dupload(T*& p, const std::vector<T>& v)
{
    cudaError_t e = dalloc(p, v.size());
    if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
    return e;
}

}  // namespace

extern "C" int lcs_forest_create(int kind, uint32_t n_scenes, const uint32_t* elem_offsets, const uint32_t* vert_offsets,
                                 lcs_forest** out)
{
    if (!out || !elem_offsets || !vert_offsets || n_scenes == 0 || (kind != LCS_TREE_EDGE && kind != LCS_TREE_FACE))
        return lcs_fail(LCS_ERR_INVALID, "lcs_forest_create: bad argument");
    if (elem_offsets[0] != 0) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_create: element offsets must start at 0");
    std::vector<uint32_t> eoff(elem_offsets, elem_offsets + n_scenes + 1), ioff(n_scenes + 1, 0),
        boff(n_scenes + 1, 0), bcover(n_scenes);
    for (uint32_t s = 0; s < n_scenes; ++s) {
        if (eoff[s + 1] < eoff[s] + 2 || vert_offsets[s + 1] < vert_offsets[s])
            return lcs_fail(LCS_ERR_INVALID, "lcs_forest_create: every scene needs at least two elements");
        const uint32_t ne = eoff[s + 1] - eoff[s];
        ioff[s + 1] = ioff[s] + ne - 1;
        const uint32_t nb = (ne + 255) / 256;
        boff[s + 1] = boff[s] + nb;
        // the reference's second pass covers ceil(n_verts / 256) partials (lbvh.cpp:958, 968)
        const uint32_t cover = (vert_offsets[s + 1] - vert_offsets[s] + 255) / 256;
        bcover[s] = std::min(cover, nb);
    }
    lcs_forest* f = new (std::nothrow) lcs_forest();
    if (!f) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_create: out of host memory");
    f->kind = kind;
    f->S = n_scenes;
    f->N = eoff[n_scenes];
    f->NI = ioff[n_scenes];
    f->NB = boff[n_scenes];
    uint32_t sb = 0;
    while ((1ull << sb) < n_scenes) ++sb;
    f->sbits = sb;
    f->h_eoff = eoff;
    f->h_ioff = ioff;
    std::vector<uint32_t> escene(f->N), iscene(f->NI), bscene(f->NB);
    for (uint32_t s = 0; s < n_scenes; ++s) {
        std::fill(escene.begin() + eoff[s], escene.begin() + eoff[s + 1], s);
        std::fill(iscene.begin() + ioff[s], iscene.begin() + ioff[s + 1], s);
        std::fill(bscene.begin() + boff[s], bscene.begin() + boff[s + 1], s);
    }
    const size_t nodes = (size_t)f->NI + f->N;
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(dupload(f->eoff, eoff));
    A(dupload(f->ioff, ioff));
    A(dupload(f->boff, boff));
    A(dupload(f->bcover, bcover));
    A(dupload(f->escene, escene));
    A(dupload(f->iscene, iscene));
    A(dupload(f->bscene, bscene));
    A(dalloc(f->centers, f->N));
    A(dalloc(f->block_aabb, 6 * (size_t)f->NB));
    A(dalloc(f->gaabb, 6 * (size_t)n_scenes));
    A(dalloc(f->m30, f->N));
    A(dalloc(f->keys, f->N));
    A(dalloc(f->keys_alt, f->N));
    A(dalloc(f->vals, f->N));
    A(dalloc(f->vals_alt, f->N));
    A(dalloc(f->hist, rs::hist_words(f->N)));
    A(dalloc(f->ms64, f->N));
    A(dalloc(f->parent, nodes));
    A(dalloc(f->children, nodes));
    A(dalloc(f->slot, nodes));
    A(dalloc(f->wide, 4 * (size_t)f->NI));
    A(dalloc(f->counters, f->NI));
    A(dalloc(f->healthy, 1));
    A(dalloc(f->saved_count, 1));
    if (e == cudaSuccess) e = cudaMemset(f->counters, 0, sizeof(uint32_t) * (size_t)f->NI);
    if (e == cudaSuccess) e = cudaMemset(f->wide, 0, sizeof(float4) * 4 * (size_t)f->NI);
    if (e != cudaSuccess) {
        lcs_forest_destroy(f);
        return lcs_fail(LCS_ERR_CUDA, "lcs_forest_create: allocation failed");
    }
    f->sgo = f->vals;
    f->skeys = f->keys;
    *out = f;
    return LCS_OK;
}

extern "C" int lcs_forest_destroy(lcs_forest* f)
{
    if (!f) return LCS_OK;
    void* ptrs[] = {f->eoff, f->ioff, f->boff, f->bcover, f->escene, f->iscene, f->bscene, f->centers,
                    f->block_aabb, f->gaabb, f->m30, f->keys, f->keys_alt, f->vals, f->vals_alt, f->hist,
                    f->ms64, f->parent, f->children, f->slot, f->wide, f->counters, f->healthy, f->saved_count};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete f;
    return LCS_OK;
}

extern "C" int lcs_forest_build(lcs_forest* f, const float* x, const uint32_t* elems, lcs_stream stream)
{
    if (!f || !x || !elems) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_build: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const float4* X = reinterpret_cast<const float4*>(x);
    k_f_pass1<<<f->NB, 256, 0, s>>>(f->kind, X, elems, f->eoff, f->boff, f->bscene, f->centers, f->block_aabb);
    lcs_count_launch();
    k_f_pass2<<<f->S, 256, 0, s>>>(f->block_aabb, f->boff, f->bcover, f->gaabb);
    lcs_count_launch();
    const int g = grid_for(f->N, 256);
    k_f_mortons<<<g, 256, 0, s>>>(f->centers, f->gaabb, f->escene, f->N, f->m30, f->keys, f->vals);
    lcs_count_launch();
    const bool alt = rs::sort_pairs<uint64_t>(f->keys, f->vals, f->keys_alt, f->vals_alt, nullptr, f->N, f->N, 0,
                                              30 + (int)f->sbits, f->hist, s);
    f->sgo = alt ? f->vals_alt : f->vals;
    f->skeys = alt ? f->keys_alt : f->keys;
    k_f_apply<<<g, 256, 0, s>>>(f->skeys, f->sgo, f->escene, f->eoff, f->ioff, f->N, f->NI, f->ms64, f->children,
                                f->parent, f->healthy);
    lcs_count_launch();
    const int gi = grid_for(f->NI, 256);
    k_f_build_inner<<<gi, 256, 0, s>>>(f->ms64, f->sgo, f->iscene, f->eoff, f->ioff, f->NI, f->parent, f->children,
                                       f->slot, f->wide);
    lcs_count_launch();
    k_f_check<<<gi, 256, 0, s>>>(f->children, f->parent, f->NI, f->healthy);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    f->built = true;
    return LCS_OK;
}

extern "C" int lcs_forest_update_refit(lcs_forest* f, const float* thickness, const float* x0, const float* x1,
                                       const uint32_t* elems, lcs_stream stream)
{
    if (!f || !thickness || !x0 || !x1 || !elems) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_update_refit: bad argument");
    // the sorted order and the slots are written by the build: before it they hold no valid indices
    if (!f->built) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_update_refit: the forest has not been built");
    k_f_refit<<<grid_for(f->N, 256), 256, 0, (cudaStream_t)stream>>>(
        f->kind, f->N, f->NI, f->sgo, f->slot, f->parent, thickness, reinterpret_cast<const float4*>(x0),
        reinterpret_cast<const float4*>(x1), elems, f->wide, f->counters, f->healthy);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

// The traversal's launch shape (threads per block: 64, 128 or 256; the grid covers every query, at most 2048
// threads per SM) is tuned on the first query of a forest: the query runs once in each shape, timed with CUDA
// events, with the candidate count restored before each run, so that the last run's pairs are the result
// (every run writes the same set).  Later queries use the fastest shape.
template <bool EE>
static int f_query_tuned(const lcs_forest* f, uint32_t n_queries, const uint32_t* qscene, const float4* x0,
                         const float4* x1, const uint2* edges, const float* d_hat, const float* thickness, uint2* pairs,
                         uint32_t capacity, uint32_t* d_count, const uint32_t* order, uint32_t* capped,
                         const uint8_t* only, cudaStream_t s)
{
    auto launch = [&](uint32_t threads) {
        k_f_query<EE><<<grid_for(n_queries, (int)threads, (int)(2048u / threads)), threads, 0, s>>>(
            f->wide, f->ioff, qscene, x0, x1, edges, n_queries, d_hat, thickness, pairs, capacity, d_count, order,
            capped, only);
        lcs_count_launch();
    };
    if (f->q_threads != 0) {
        launch(f->q_threads);
        LCS_LAUNCH_CHECK();
        return LCS_OK;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        if (e0) cudaEventDestroy(e0);
        f->q_threads = 128;  // untuned default
        launch(f->q_threads);
        LCS_LAUNCH_CHECK();
        return LCS_OK;
    }
    int rc = LCS_OK;
    float best = 0.0f;
    uint32_t best_threads = 128;
    if (cudaMemcpyAsync(f->saved_count, d_count, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        rc = LCS_ERR_CUDA;
    for (uint32_t threads : {64u, 256u, 128u}) {
        if (rc != LCS_OK) break;
        if (cudaMemcpyAsync(d_count, f->saved_count, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaEventRecord(e0, s) != cudaSuccess) {
            rc = LCS_ERR_CUDA;
            break;
        }
        launch(threads);
        float ms = 0.0f;
        if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = LCS_ERR_CUDA;
            break;
        }
        if (best == 0.0f || ms < best) {
            best = ms;
            best_threads = threads;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != LCS_OK) return lcs_fail(rc, "lcs_forest_query: tuning the launch shape failed");
    f->q_threads = best_threads;
    f->q_ms = best;
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_forest_query_tuning(const lcs_forest* f, uint32_t* threads_per_block, float* query_ms)
{
    if (!f) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_query_tuning: null handle");
    if (threads_per_block) *threads_per_block = f->q_threads;
    if (query_ms) *query_ms = f->q_ms;
    return LCS_OK;
}

extern "C" int lcs_forest_query_vf(const lcs_forest* face_forest, const float* x0, const float* x1, uint32_t n_verts,
                                   const uint32_t* vert_scene, const float* d_hat, const float* thickness,
                                   uint32_t* pairs, uint32_t capacity, uint32_t* d_count, lcs_stream stream)
{
    return lcs_forest_query_vf_capped(face_forest, x0, x1, n_verts, vert_scene, d_hat, thickness, pairs, capacity,
                                      d_count, nullptr, stream);
}

int lcs_forest_query_vf_capped(const lcs_forest* face_forest, const float* x0, const float* x1, uint32_t n_verts,
                               const uint32_t* vert_scene, const float* d_hat, const float* thickness, uint32_t* pairs,
                               uint32_t capacity, uint32_t* d_count, uint32_t* capped, lcs_stream stream,
                               const uint8_t* only)
{
    const lcs_forest* f = face_forest;
    if (!f || f->kind != LCS_TREE_FACE || !x0 || !x1 || !vert_scene || !d_hat || !thickness || !d_count ||
        (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_forest_query_vf: bad argument");
    if (n_verts == 0) return LCS_OK;
    if (!f->built) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_query_vf: the forest has not been built");
    return f_query_tuned<false>(f, n_verts, vert_scene, reinterpret_cast<const float4*>(x0),
                                reinterpret_cast<const float4*>(x1), nullptr, d_hat, thickness,
                                reinterpret_cast<uint2*>(pairs), capacity, d_count, nullptr, capped, only,
                                (cudaStream_t)stream);
}

extern "C" int lcs_forest_query_ee(const lcs_forest* edge_forest, const float* x0, const float* x1,
                                   const uint32_t* edges, const float* d_hat, const float* thickness, uint32_t* pairs,
                                   uint32_t capacity, uint32_t* d_count, lcs_stream stream)
{
    return lcs_forest_query_ee_capped(edge_forest, x0, x1, edges, d_hat, thickness, pairs, capacity, d_count, nullptr,
                                      stream);
}

int lcs_forest_query_ee_capped(const lcs_forest* edge_forest, const float* x0, const float* x1, const uint32_t* edges,
                               const float* d_hat, const float* thickness, uint32_t* pairs, uint32_t capacity,
                               uint32_t* d_count, uint32_t* capped, lcs_stream stream, const uint8_t* only)
{
    const lcs_forest* f = edge_forest;
    if (!f || f->kind != LCS_TREE_EDGE || !x0 || !x1 || !edges || !d_hat || !thickness || !d_count ||
        (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_forest_query_ee: bad argument");
    if (!f->built) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_query_ee: the forest has not been built");
    return f_query_tuned<true>(f, f->N, f->escene, reinterpret_cast<const float4*>(x0),
                               reinterpret_cast<const float4*>(x1), reinterpret_cast<const uint2*>(edges), d_hat,
                               thickness, reinterpret_cast<uint2*>(pairs), capacity, d_count, f->sgo, capped, only,
                               (cudaStream_t)stream);
}

extern "C" int lcs_forest_health(lcs_forest* f, int* healthy, lcs_stream stream)
{
    if (!f || !healthy) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_health: bad argument");
    uint32_t h = 0;
    LCS_CUDA_TRY(cudaMemcpyAsync(&h, f->healthy, 4, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    LCS_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    *healthy = (int)h;
    return LCS_OK;
}

extern "C" int lcs_forest_export_scene(const lcs_forest* f, uint32_t scene, uint32_t* parent, uint32_t* children,
                                       uint32_t* object_idx, uint64_t* morton_sorted, uint32_t* sorted_get_original,
                                       float* node_aabb, float* global_aabb6, lcs_stream stream)
{
    if (!f || scene >= f->S) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_export_scene: bad argument");
    if (!f->built) return lcs_fail(LCS_ERR_INVALID, "lcs_forest_export_scene: the forest has not been built");
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n = f->h_eoff[scene + 1] - f->h_eoff[scene];
    const ForestView v{f->eoff, f->ioff, f->parent, f->slot, f->sgo, f->children, f->ms64, f->wide, f->NI};
    k_f_export<<<grid_for(2 * (uint64_t)n - 1, 256), 256, 0, s>>>(v, scene, parent, reinterpret_cast<uint2*>(children),
                                                                   object_idx, morton_sorted, sorted_get_original,
                                                                   node_aabb);
    lcs_count_launch();
    if (global_aabb6)
        LCS_CUDA_TRY(cudaMemcpyAsync(global_aabb6, f->gaabb + 6 * (size_t)scene, 24, cudaMemcpyDeviceToDevice, s));
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}
