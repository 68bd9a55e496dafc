// lbvh.cu -- LBVH over vertices, edges or faces: build, refit and broad-phase traversal.
//
// Follows Solver/CollisionDetector/lbvh.cpp of the reference (citations per kernel) with a
// B200 layout for traversal: every inner node is one 64-byte record holding the boxes of
// both children, {min.xyz | child code}, {max.xyz}, {min.xyz | child code}, {max.xyz}, where
// a child code is the inner node index, or 0x80000000 | element id for a leaf.  One
// traversal step is therefore one 64-byte load instead of the reference's three dependent
// loads (children, child AABB, object_idx).  The reference's LbvhData layout is produced on
// demand by lcs_bvh_export for tests and interop.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "lcs_common.cuh"
#include "lbvh_common.cuh"
#include "lcs_internal.h"
#include "radix_sort.cuh"
#include "scan.cuh"

using namespace lcs;

struct lcs_bvh {
    int kind = 0;
    uint32_t n = 0, ni = 0, nb = 0;  // leaves, inner nodes, 256-element blocks
    float4* centers = nullptr;       // n
    float* block_aabb = nullptr;     // 6 * nb
    float* gaabb = nullptr;          // 6
    uint32_t* m30 = nullptr;         // n, unsorted 30-bit Morton codes
    uint32_t* keys = nullptr;        // n, sort buffers
    uint32_t* keys_alt = nullptr;
    uint32_t* vals = nullptr;
    uint32_t* vals_alt = nullptr;
    uint32_t* hist = nullptr;
    uint32_t* sgo = nullptr;         // sorted_get_original (points into vals or vals_alt)
    uint32_t* m30_sorted = nullptr;  // (points into keys or keys_alt)
    uint64_t* ms64 = nullptr;        // n, sorted morton64 = m30 << 32 | element id
    uint32_t* parent = nullptr;      // 2n - 1
    uint2* children = nullptr;       // 2n - 1, reference layout
    uint32_t* slot = nullptr;        // 2n - 1, 2 * parent + side
    float4* wide = nullptr;          // 4 * max(ni, 1)
    float4* wide4 = nullptr;         // 8 * max(ni, 1): 4-child records of the even-depth inner nodes
    uint8_t* even = nullptr;         // max(ni, 1): inner node at even depth (root: depth 0)
    // the refit's tables, rebuilt with the topology (see k_eorder)
    uint2* range = nullptr;          // max(ni, 1): sorted leaf positions [first, last] under each inner node
    uint32_t* swap_diff = nullptr;   // n + 1: +1 / -1 at the ends of each swapped node's left range
    uint32_t* swap_cov = nullptr;    // n + 1: its exclusive prefix sum
    uint32_t* scan_tmp = nullptr;
    uint32_t* n_plus_1 = nullptr;    // 1: n + 1, the scan's element count
    uint32_t* leaf_at = nullptr;     // n: sorted leaf position at each position of the union order
    uint32_t* node_at = nullptr;     // max(ni, 1): inner node whose two children meet after each position
    uint4* order_range = nullptr;    // max(ni, 1): {first, last} union-order positions, last sorted position
    uint32_t* spans = nullptr;       // max(ni, 1): inner nodes whose leaves lie in more than one refit chunk
    uint32_t* span_count = nullptr;  // 1
    float4* seg_box = nullptr;       // 2 per 32 union-order positions (whole refit chunks): {min | 0}{max | 0}
    float4* chunk_box = nullptr;     // 2 per refit chunk: its union
    uint32_t* healthy = nullptr;     // 1
    uint32_t* maxdepth = nullptr;    // 1: depth of the deepest inner node (root: 0), capped at 256
    bool built = false;              // a construct has written the topology, slots and refit tables
};

namespace {

// fn_reduce_{vert,edge,face}_tree_global_aabb, lbvh.cpp:449-491: centres + per-256 partials
__global__ void __launch_bounds__(256) k_reduce_pass1(int kind, const float4* __restrict__ x,
                                                      const uint32_t* __restrict__ elems, uint32_t n,
                                                      float4* __restrict__ centers, float* __restrict__ block_aabb)
{
    __shared__ float red[8][6];
    const uint32_t e = blockIdx.x * 256 + threadIdx.x;
    v3 mn = mk3(INFINITY, INFINITY, INFINITY), mx = mk3(-INFINITY, -INFINITY, -INFINITY);
    if (e < n) {
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

// fn_reduce_aabb_2_pass(_atomic), lbvh.cpp:396-447, over the first nb_cover partials
__global__ void __launch_bounds__(256) k_reduce_pass2(const float* __restrict__ block_aabb, uint32_t nb_cover,
                                                      float* __restrict__ gaabb)
{
    __shared__ float red[8][6];
    float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (uint32_t b = threadIdx.x; b < nb_cover; b += 256)
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = k < 3 ? fmn(v[k], block_aabb[6 * b + k]) : fmx(v[k], block_aabb[6 * b + k]);
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
        gaabb[threadIdx.x] = r;
    }
}

// fn_compute_mortons, lbvh.cpp:507-523 (30-bit code; the element id is the sort value)
__global__ void k_mortons(const float4* __restrict__ centers, const float* __restrict__ gaabb, uint32_t n,
                          uint32_t* __restrict__ m30, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
    const float inv0 = 1.0f / fmx(gaabb[3] - gaabb[0], 1e-6f);
    const float inv1 = 1.0f / fmx(gaabb[4] - gaabb[1], 1e-6f);
    const float inv2 = 1.0f / fmx(gaabb[5] - gaabb[2], 1e-6f);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = centers[i];
        uint32_t m = morton32((c.x - gaabb[0]) * inv0, (c.y - gaabb[1]) * inv1, (c.z - gaabb[2]) * inv2);
        m30[i] = m;
        keys[i] = m;
        vals[i] = i;
    }
}

// fn_reset_tree + fn_apply_sorted, lbvh.cpp:493-539
__global__ void k_apply_sorted(const uint32_t* __restrict__ m30s, const uint32_t* __restrict__ sgo, uint32_t n,
                               uint64_t* __restrict__ ms64, uint2* __restrict__ children, uint32_t* __restrict__ parent,
                               uint32_t* __restrict__ healthy)
{
    const uint32_t ni = n - 1;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t o = sgo[i];
        ms64[i] = ((uint64_t)m30s[i] << 32) | (uint64_t)o;
        children[ni + i] = make_uint2(o, o);
        if (i == 0) {
            parent[0] = kInvalid;
            *healthy = 1u;
        }
    }
}

// union-order positions per block of the chunked refit (k_refit_chunks); a multiple of 32
constexpr uint32_t kRefitChunk = 512;
constexpr uint32_t kRefitSegs = kRefitChunk / 32;  // 32-position segments per chunk
constexpr int kRefitLevels = 4;                    // sparse-table levels over a chunk's segments (2^4 = 16)
static_assert((1u << kRefitLevels) == kRefitSegs, "one sparse-table level per doubling of the segment count");

// fn_build_inner_nodes with determineRange / findSplit, lbvh.cpp:204-291, 541-596; also the
// traversal records' child codes, the child -> parent slot map, each inner node's sorted leaf range and,
// for a node whose right child is a leaf (put first in the reference's child layout), +1 / -1 at the ends of
// its left child's range in swap_diff (see k_eorder)
__global__ void k_build_inner(const uint64_t* __restrict__ ms, const uint32_t* __restrict__ sgo, uint32_t n,
                              uint32_t* __restrict__ parent, uint2* __restrict__ children,
                              uint32_t* __restrict__ slot, float4* __restrict__ wide, uint32_t* __restrict__ maxdepth,
                              uint2* __restrict__ range, uint32_t* __restrict__ swap_diff)
{
    const int ni = (int)n - 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) *maxdepth = 0u;  // raised by k_depth_parity, launched after this
    for (int nid = blockIdx.x * blockDim.x + threadIdx.x; nid < ni; nid += gridDim.x * blockDim.x) {
        int i = 0, j = ni;
        if (nid != 0) {
            const uint64_t mi = ms[nid];
            const int cl = __clzll((long long)(mi ^ ms[nid - 1]));
            const int cr = __clzll((long long)(mi ^ ms[nid + 1]));
            const int d = cl < cr ? 1 : -1;
            const int cp_min = cl < cr ? cl : cr;
            int lmax = 2;
            while (cp_ij(mi, nid + lmax * d, ms, (int)n) > cp_min) lmax <<= 1;
            int l = 0;
            for (int t = lmax >> 1; t >= 1; t >>= 1)
                if (cp_ij(mi, nid + (l + t) * d, ms, (int)n) > cp_min) l += t;
            i = nid;
            j = nid + l * d;
        }
        int a = i < j ? i : j, b = i < j ? j : i;
        range[nid] = make_uint2((uint32_t)a, (uint32_t)b);
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
        if (cright >= ni) {  // the right child is the leaf b: it becomes the first child
            atomicAdd(&swap_diff[a], 1u);
            atomicAdd(&swap_diff[b], 0xFFFFFFFFu);
            int t = cleft;
            cleft = cright;
            cright = t;
        }
        parent[cleft] = (uint32_t)nid;
        parent[cright] = (uint32_t)nid;
        children[nid] = make_uint2((uint32_t)cleft, (uint32_t)cright);
        slot[cleft] = 2u * (uint32_t)nid + 0u;
        slot[cright] = 2u * (uint32_t)nid + 1u;
        const uint32_t code_l = cleft < ni ? (uint32_t)cleft : (0x80000000u | sgo[cleft - ni]);
        const uint32_t code_r = cright < ni ? (uint32_t)cright : (0x80000000u | sgo[cright - ni]);
        wide[4 * nid + 0].w = __uint_as_float(code_l);
        wide[4 * nid + 2].w = __uint_as_float(code_r);
    }
}

// 4-wide traversal records.  The binary tree stays the reference's (topology, refit and export are
// bit-exact against it); during each refit every inner node b at even depth gets a record of its four
// grandchild slots (a leaf child keeps its own slot), written once its children's slots are final (by the
// chunk kernel of the refit for nodes inside one chunk, else by k_refit_span_records):
// {min.xyz | code}{max.xyz | last} x 4, 128 B, empty slots as inverted boxes that no strict
// overlap test passes.  A traversal then takes one dependent
// 128-B fetch where the binary walk took two 64-B ones.  k_depth_parity marks the even-depth inner nodes
// after each build (a climb to the root per node, at most 256 levels).
__global__ void k_depth_parity(const uint32_t* __restrict__ parent, uint32_t ni, uint8_t* __restrict__ even,
                               uint32_t* __restrict__ maxdepth)
{
    uint32_t deepest = 0;
    for (uint32_t nid = blockIdx.x * blockDim.x + threadIdx.x; nid < ni; nid += gridDim.x * blockDim.x) {
        uint32_t p = nid, d = 0;
        while (p != 0u && p < ni && d < 256u) {
            p = parent[p];
            ++d;
        }
        even[nid] = (d & 1u) == 0u ? 1 : 0;
        deepest = d > deepest ? d : deepest;
    }
    deepest = __reduce_max_sync(0xFFFFFFFFu, deepest);
    if (lane_id() == 0 && deepest) atomicMax(maxdepth, deepest);
}

// the 4-wide record of inner node b from the binary records (leaf_only: a one-leaf tree, whose two slots
// are both the leaf)
__device__ __forceinline__ void collapse_node(const float4* wide, uint32_t b, bool leaf_only, float4* wide4)
{
    float4* out = wide4 + 8 * b;
    int k = 0;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const float4 mn = __ldcg(wide + 4 * b + 2 * side), mx = __ldcg(wide + 4 * b + 2 * side + 1);
        const uint32_t code = __float_as_uint(mn.w);
        if (leaf_only || (code & 0x80000000u)) {
            __stcg(out + k, mn);
            __stcg(out + k + 1, mx);
            k += 2;
        } else {
            const float4* c = wide + 4 * code;
            const float4 c0 = __ldcg(c), c1 = __ldcg(c + 1), c2 = __ldcg(c + 2), c3 = __ldcg(c + 3);
            __stcg(out + k, c0);
            __stcg(out + k + 1, c1);
            __stcg(out + k + 2, c2);
            __stcg(out + k + 3, c3);
            k += 4;
        }
    }
    const float inf = __int_as_float(0x7f800000);
    for (; k < 8; k += 2) {
        __stcg(out + k, make_float4(inf, inf, inf, __uint_as_float(0x80000000u)));
        __stcg(out + k + 1, make_float4(-inf, -inf, -inf, __uint_as_float(0u)));
    }
}

// pairs of this traversal step (up to 4 per thread) appended with one atomic per warp: the counts' bits
// are balloted, so every lane's offset is a sum of popcounts
__device__ __forceinline__ void emit_pairs(const uint2* hit, uint32_t nhit, uint2* pairs, uint32_t capacity,
                                           uint32_t* d_count)
{
    const uint32_t active = __activemask();
    const uint32_t lt = (1u << lane_id()) - 1u;
    const uint32_t b0 = __ballot_sync(active, nhit & 1u), b1 = __ballot_sync(active, nhit & 2u),
                   b2 = __ballot_sync(active, nhit & 4u);
    const uint32_t total = __popc(b0) + 2u * __popc(b1) + 4u * __popc(b2);
    const uint32_t leader = __ffs(active) - 1;
    uint32_t base = 0;
    if (lane_id() == leader && total) base = atomicAdd(d_count, total);
    base = __shfl_sync(active, base, leader) + __popc(b0 & lt) + 2u * __popc(b1 & lt) + 4u * __popc(b2 & lt);
    for (uint32_t k = 0; k < nhit; ++k)
        if (base + k < capacity) pairs[base + k] = hit[k];
}

// fn_check_construction, lbvh.cpp:598-611
__global__ void k_check(const uint2* __restrict__ children, const uint32_t* __restrict__ parent, uint32_t ni,
                        uint32_t* __restrict__ healthy)
{
    const uint32_t nodes = 2 * ni + 1;
    for (uint32_t nid = blockIdx.x * blockDim.x + threadIdx.x; nid < ni; nid += gridDim.x * blockDim.x) {
        uint2 c = children[nid];
        // a child index outside the tree is unhealthy too (and is not followed)
        if (c.x >= nodes || c.y >= nodes || parent[c.x] != nid || parent[c.y] != nid) *healthy = 0u;
    }
}

__global__ void k_set_healthy(uint32_t* healthy) { *healthy = 1u; }

// The union order of the refit.  The reference's walk makes each inner box fmin / fmax of its children's in
// the child layout's order: left then right, except where the right child is a leaf, which k_build_inner puts
// first.  A node's box is then the fold of its leaves' boxes in the in-order sequence of the tree taken in
// layout order, and those positions have a closed form: a leaf at sorted position p moves one place later
// for every swapped ancestor whose left child holds it -- cov(p), the number of left ranges [a, b - 1] of
// swapped nodes containing p, a prefix sum of swap_diff -- and the swapped leaf b of a node [a, b] goes to
// the front of it, to a + cov(b); an inner node [a, b] holds the positions a + cov(b) .. a + cov(b) + b - a.
// Each inner node also gets the position after which its two children meet (one node per position
// 0 .. n - 2), so that a refit block finds the nodes of its chunk, and the nodes whose positions cross a
// chunk boundary are listed (in any order: each is refitted on its own).
__global__ void k_eorder(uint32_t n, const uint32_t* __restrict__ parent, const uint2* __restrict__ children,
                         const uint2* __restrict__ range, const uint32_t* __restrict__ cov_excl,
                         uint32_t* __restrict__ leaf_at, uint32_t* __restrict__ node_at,
                         uint4* __restrict__ order_range, uint32_t* __restrict__ spans, uint32_t* span_count)
{
    const uint32_t ni = n - 1;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n + ni; k += gridDim.x * blockDim.x) {
        if (k < n) {
            const uint32_t P = parent[ni + k];
            const uint2 r = range[P];
            const bool front = children[P].x == ni + k && k == r.y;
            const uint32_t pos = (front ? r.x : k) + cov_excl[k + 1];
            if (pos < n) leaf_at[pos] = k;
        } else {
            const uint32_t i = k - n;
            const uint2 r = range[i];
            const uint32_t first = r.x + cov_excl[r.y + 1], last = first + (r.y - r.x);
            const uint32_t c0 = children[i].x;
            const uint32_t size0 = c0 >= ni ? 1u : range[c0].y - range[c0].x + 1u;
            if (first + size0 - 1 < ni) node_at[first + size0 - 1] = i;
            order_range[i] = make_uint4(first, last, r.y, 0u);
            if (first / kRefitChunk != last / kRefitChunk) spans[atomicAdd(span_count, 1u)] = i;
        }
    }
}

// fn_update_*_tree_leave_aabb_v2 (lbvh.cpp:617-683) alone: the leaf slots (a one-leaf tree also gets its
// 4-wide record, both of whose slots are the leaf)
__device__ __forceinline__ void collapse_node(const float4* wide, uint32_t b, bool leaf_only, float4* wide4);

__global__ void k_leaves(int kind, uint32_t n, const uint32_t* __restrict__ sgo, const uint32_t* __restrict__ slot,
                         const float* __restrict__ thickness, const float4* __restrict__ x0,
                         const float4* __restrict__ x1, const uint32_t* __restrict__ elems, float4* wide,
                         float4* __restrict__ wide4)
{
    const uint32_t ni = n - 1;
    for (uint32_t lid = blockIdx.x * blockDim.x + threadIdx.x; lid < n; lid += gridDim.x * blockDim.x) {
        const uint32_t e = sgo[lid];
        v3 mn, mx;
        leaf_box(kind, e, thickness, x0, x1, elems, mn, mx);
        if (n == 1) {
            store_slot(wide, 0, mn, mx, 0x80000000u | e);
            store_slot(wide, 1, mn, mx, 0x80000000u | e);
            collapse_node(wide, 0, true, wide4);
        } else {
            store_slot(wide, slot[ni + lid], mn, mx, 0x80000000u | e, lid);
        }
    }
}

// fn_refit_tree_aabb (lbvh.cpp:702-754) without its bottom-up walk.  The walk makes every inner box the
// union of its children's, fmin / fmax of the form `a < b ? a : b` in the child layout's order; over the
// leaves of a node that is the fold of their boxes in the union order (k_eorder), and since that operation
// is associative and idempotent on everything but NaN (it keeps the later of equal extremes, +0 / -0
// included), any split of a node's union-order range into pieces combined in order -- overlapping pieces
// too -- gives the same bits.  So every inner box is computed straight from its range of leaves in union
// order, with no serial climb; "chunks" and "segments" below are runs of union-order positions:
//   * k_refit_chunks: one block per kRefitChunk positions keeps their leaves' boxes, the prefix and suffix
//     unions of each 32-position segment (warp scans) and a sparse table over the segment unions in shared
//     memory; every inner node whose range lies in the chunk is then one segment's fold, or a suffix, at
//     most two overlapping sparse-table entries and a prefix.  It writes the segment and chunk unions and,
//     after a block barrier, the 4-wide records of its even-depth nodes.
//   * k_refit_spans: one warp per node whose range crosses a chunk boundary (listed by k_eorder): leaves
//     of the first and last segment, segments of the first and last chunk and whole chunks in between,
//     each piece reduced across the warp in lane order.
//   * k_refit_span_records: the 4-wide records of the crossing nodes at even depth.
// NaN coordinates (a diverged state, reported by the solver) may give other bits than the walk does.

__device__ __forceinline__ void box_id(float (&v)[6])
{
    v[0] = v[1] = v[2] = __int_as_float(0x7f800000);
    v[3] = v[4] = v[5] = __int_as_float(0xff800000);
}

// l = l (on the left) joined with r (on the right)
__device__ __forceinline__ void box_join(float (&l)[6], const float (&r)[6])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) l[c] = fmn(l[c], r[c]);
#pragma unroll
    for (int c = 3; c < 6; ++c) l[c] = fmx(l[c], r[c]);
}

// the lanes' pieces joined in lane order (lane 0 holds the result): pieces of 1, 2, 4, ... lanes
__device__ __forceinline__ void box_warp_fold(float (&v)[6])
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        float o[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) o[c] = __shfl_down_sync(0xFFFFFFFFu, v[c], d);
        if ((lane_id() & (2 * d - 1)) == 0) box_join(v, o);
    }
}

__device__ __forceinline__ void box_ld(const float4* p, float (&v)[6])
{
    const float4 mn = __ldcg(p), mx = __ldcg(p + 1);
    v[0] = mn.x; v[1] = mn.y; v[2] = mn.z;
    v[3] = mx.x; v[4] = mx.y; v[5] = mx.z;
}

__global__ void __launch_bounds__(kRefitChunk) k_refit_chunks(
    int kind, uint32_t n, const uint32_t* __restrict__ sgo, const uint32_t* __restrict__ slot,
    const uint32_t* __restrict__ leaf_at, const uint32_t* __restrict__ node_at,
    const uint4* __restrict__ order_range, const uint8_t* __restrict__ even, const float* __restrict__ thickness,
    const float4* __restrict__ x0, const float4* __restrict__ x1, const uint32_t* __restrict__ elems, int write_leaf,
    float4* wide, float4* __restrict__ wide4, float4* __restrict__ seg_box, float4* __restrict__ chunk_box)
{
    __shared__ float s_leaf[6][kRefitChunk], s_pre[6][kRefitChunk], s_suf[6][kRefitChunk];
    __shared__ float s_tab[kRefitLevels][6][kRefitSegs];  // s_tab[k][.][s]: segments s .. s + 2^k - 1
    const uint32_t ni = n - 1, t = threadIdx.x, lane = t & 31u, w = t >> 5;
    const uint32_t c0 = blockIdx.x * kRefitChunk, pos = c0 + t;
    float b[6];
    box_id(b);
    if (pos < n) {
        const uint32_t lid = __ldg(&leaf_at[pos]);
        const uint32_t sl = slot[ni + lid];
        if (write_leaf) {
            const uint32_t e = sgo[lid];
            v3 mn, mx;
            leaf_box(kind, e, thickness, x0, x1, elems, mn, mx);
            store_slot(wide, sl, mn, mx, 0x80000000u | e, lid);
            b[0] = mn.x; b[1] = mn.y; b[2] = mn.z;
            b[3] = mx.x; b[4] = mx.y; b[5] = mx.z;
        } else {
            box_ld(wide + 4 * (sl >> 1) + 2 * (sl & 1u), b);
        }
    }
    float pre[6], suf[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) pre[c] = suf[c] = b[c];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        float up[6], dn[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            up[c] = __shfl_up_sync(0xFFFFFFFFu, pre[c], d);
            dn[c] = __shfl_down_sync(0xFFFFFFFFu, suf[c], d);
        }
        if (lane >= (uint32_t)d) {  // lanes lane - 2d + 1 .. lane - d, then this piece
            box_join(up, pre);
#pragma unroll
            for (int c = 0; c < 6; ++c) pre[c] = up[c];
        }
        if (lane + d < 32u) box_join(suf, dn);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        s_leaf[c][t] = b[c];
        s_pre[c][t] = pre[c];
        s_suf[c][t] = suf[c];
    }
    if (lane == 31u) {
#pragma unroll
        for (int c = 0; c < 6; ++c) s_tab[0][c][w] = pre[c];
        float4* o = seg_box + 2 * (c0 / 32u + w);
        __stcg(o, make_float4(pre[0], pre[1], pre[2], 0.0f));
        __stcg(o + 1, make_float4(pre[3], pre[4], pre[5], 0.0f));
    }
    __syncthreads();
    if (w == 0) {
        float v[6];
        if (lane < kRefitSegs) {
#pragma unroll
            for (int c = 0; c < 6; ++c) v[c] = s_tab[0][c][lane];
        } else {
            box_id(v);
        }
        float all[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) all[c] = v[c];
#pragma unroll
        for (int k = 1; k < kRefitLevels; ++k) {
            float o[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) o[c] = __shfl_down_sync(0xFFFFFFFFu, v[c], 1 << (k - 1));
            box_join(v, o);  // entries whose window runs past the chunk are never read
            if (lane < kRefitSegs) {
#pragma unroll
                for (int c = 0; c < 6; ++c) s_tab[k][c][lane] = v[c];
            }
        }
        box_warp_fold(all);
        if (lane == 0) {
            __stcg(chunk_box + 2 * blockIdx.x, make_float4(all[0], all[1], all[2], 0.0f));
            __stcg(chunk_box + 2 * blockIdx.x + 1, make_float4(all[3], all[4], all[5], 0.0f));
        }
    }
    __syncthreads();
    bool mine = false;
    uint32_t node = 0;
    if (pos < ni) {
        node = __ldg(&node_at[pos]);
        const uint4 r = __ldg(&order_range[node]);
        if (r.x >= c0 && r.y < c0 + kRefitChunk) {
            mine = true;
            const uint32_t la = r.x - c0, lb = r.y - c0, sa = la >> 5, sb = lb >> 5;
            float v[6];
            if (sa == sb) {
                box_id(v);
                for (uint32_t j = la; j <= lb; ++j) {
                    float o[6];
#pragma unroll
                    for (int c = 0; c < 6; ++c) o[c] = s_leaf[c][j];
                    box_join(v, o);
                }
            } else {
                float o[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) v[c] = s_suf[c][la];
                if (sb > sa + 1) {
                    const uint32_t len = sb - sa - 1;
                    const int k = 31 - __clz((int)len);
#pragma unroll
                    for (int c = 0; c < 6; ++c) o[c] = s_tab[k][c][sa + 1];
                    box_join(v, o);
#pragma unroll
                    for (int c = 0; c < 6; ++c) o[c] = s_tab[k][c][sb - (1u << k)];
                    box_join(v, o);
                }
#pragma unroll
                for (int c = 0; c < 6; ++c) o[c] = s_pre[c][lb];
                box_join(v, o);
            }
            if (node != 0) store_slot(wide, slot[node], mk3(v[0], v[1], v[2]), mk3(v[3], v[4], v[5]), node, r.z);
        }
    }
    __syncthreads();  // the chunk's slots are written: its nodes' children records are final
    if (mine && even[node]) collapse_node(wide, node, false, wide4);
}

__global__ void __launch_bounds__(256) k_refit_spans(uint32_t n, const uint32_t* __restrict__ spans,
                                                     const uint32_t* __restrict__ span_count,
                                                     const uint4* __restrict__ order_range,
                                                     const uint32_t* __restrict__ leaf_at, const uint32_t* __restrict__ slot,
                                                     const float4* __restrict__ seg_box,
                                                     const float4* __restrict__ chunk_box, float4* wide)
{
    const uint32_t ni = n - 1, lane = lane_id();
    const uint32_t cnt = *span_count;
    for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < cnt; j += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t i = spans[j];
        const uint4 r = order_range[i];
        const uint32_t a = r.x, b = r.y, ca = a / kRefitChunk, cb = b / kRefitChunk, sa = a >> 5, sb = b >> 5;
        float acc[6], v[6];
        box_id(acc);
        // 1: leaves a .. the end of segment sa (a full segment: chunk ca is not the last)
        box_id(v);
        if ((sa << 5) + lane >= a) {
            const uint32_t sl = slot[ni + leaf_at[(sa << 5) + lane]];
            box_ld(wide + 4 * (sl >> 1) + 2 * (sl & 1u), v);
        }
        box_warp_fold(v);
        box_join(acc, v);
        // 2: the segments of chunk ca after sa
        box_id(v);
        if (sa + 1 + lane < (ca + 1) * kRefitSegs) box_ld(seg_box + 2 * (sa + 1 + lane), v);
        box_warp_fold(v);
        box_join(acc, v);
        // 3: chunks ca + 1 .. cb - 1, a contiguous run per lane
        box_id(v);
        {
            const uint32_t nc = cb - ca - 1, per = (nc + 31) >> 5;
            for (uint32_t k = 0; k < per; ++k) {
                const uint32_t c = ca + 1 + lane * per + k;
                if (c < cb) {
                    float o[6];
                    box_ld(chunk_box + 2 * c, o);
                    box_join(v, o);
                }
            }
        }
        box_warp_fold(v);
        box_join(acc, v);
        // 4: the segments of chunk cb before sb
        box_id(v);
        if (cb * kRefitSegs + lane < sb) box_ld(seg_box + 2 * (cb * kRefitSegs + lane), v);
        box_warp_fold(v);
        box_join(acc, v);
        // 5: leaves of segment sb up to b
        box_id(v);
        if ((sb << 5) + lane <= b) {
            const uint32_t sl = slot[ni + leaf_at[(sb << 5) + lane]];
            box_ld(wide + 4 * (sl >> 1) + 2 * (sl & 1u), v);
        }
        box_warp_fold(v);
        box_join(acc, v);
        if (lane == 0 && i != 0)
            store_slot(wide, slot[i], mk3(acc[0], acc[1], acc[2]), mk3(acc[3], acc[4], acc[5]), i, r.z);
    }
}

__global__ void k_refit_span_records(const uint32_t* __restrict__ spans, const uint32_t* __restrict__ span_count,
                                     const uint8_t* __restrict__ even, const float4* wide, float4* __restrict__ wide4)
{
    const uint32_t cnt = *span_count;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) {
        const uint32_t i = spans[j];
        if (even[i]) collapse_node(wide, i, false, wide4);
    }
}

// query_template2 (lbvh.cpp:293-360) for fn_query_from_verts_v2 (EE = false, lbvh.cpp:776-808)
// and fn_query_from_edges_v2 (EE = true, lbvh.cpp:810-846)
constexpr int kStack4 = 64;  // entries of the 4-wide traversal stack

// The reference's stack holds at most one pending node per level above the node it pops (children are
// pushed left, right and the right one is popped next), so it can only fill -- and end a query early --
// in a tree with an inner node at depth >= 32.  k_depth_parity records the deepest inner node after each
// build; the 4-wide walks below serve the trees where that early exit cannot happen (their own 64-entry
// stack then holds at most 3 nodes per 4-wide level: 48), and k_query_ref restates the reference's walk,
// early exit included, on the others.  Each launch reads the depth and returns at once when the tree is
// the other kind, so the choice costs no host synchronisation.
constexpr uint32_t kRefStack = 32;

template <bool EE>
__global__ void __launch_bounds__(128) k_query(const float4* __restrict__ wide4, uint32_t n_leaves,
                                               const float4* __restrict__ x0, const float4* __restrict__ x1,
                                               const uint2* __restrict__ edges, uint32_t n_queries,
                                               const float* __restrict__ dhat, const float* __restrict__ thickness,
                                               uint2* __restrict__ pairs, uint32_t capacity, uint32_t* d_count,
                                               const uint32_t* __restrict__ order, uint32_t* capped,
                                               const uint32_t* __restrict__ maxdepth)
{
    if (__ldg(maxdepth) >= kRefStack) return;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_queries; t += gridDim.x * blockDim.x) {
        // queries in the order of `order` (the tree's Morton order when the queries are its own
        // leaves): neighbouring threads then walk nearly the same nodes
        const uint32_t q = order ? __ldg(&order[t]) : t;
        float box[6];
        {
            v3 mn, mx;
            uint32_t v0;
            if (EE) {
                uint2 ed = __ldg(&edges[q]);
                v3 s0 = ld3(x0, ed.x), s1 = ld3(x0, ed.y), e0 = ld3(x1, ed.x), e1 = ld3(x1, ed.y);
                mn = min3(min3(s0, s1), min3(e0, e1));
                mx = max3(max3(s0, s1), max3(e0, e1));
                v0 = ed.x;
            } else {
                v3 a = ld3(x0, q), b = ld3(x1, q);
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
        uint32_t stack[kStack4];
        int sp = 0;
        uint32_t loop = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const uint32_t node = stack[--sp];
            const float4* r = wide4 + 8 * node;
            float4 rec[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) ld_slot(r + 2 * j, rec[2 * j], rec[2 * j + 1]);
            bool stop = false;
            uint2 hit[4];
            uint32_t nhit = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float4 mn = rec[2 * k], mx = rec[2 * k + 1];
                if (!stop && overlap(mn, mx, box)) {
                    const uint32_t code = __float_as_uint(mn.w);
                    if (code & 0x80000000u) {
                        const uint32_t obj = code & 0x7FFFFFFFu;
                        if (!EE || q < obj) hit[nhit++] = make_uint2(q, obj);
                    } else if (sp < kStack4) {
                        stack[sp++] = code;
                    } else {
                        stop = true;  // a full stack ends the whole traversal (lbvh.cpp:344-351)
                    }
                }
            }
            emit_pairs(hit, nhit, pairs, capacity, d_count);
            if (stop || ++loop > 100000u) {  // the reference's early exits; reported so callers know the
                if (capped) atomicOr(capped, 1u);  // list may lack pairs a complete traversal would find
                break;
            }
        }
    }
}

// query_template2 as the reference runs it (lbvh.cpp:293-360) on the binary records, for trees with an
// inner node at depth >= 32 (see kRefStack): a stack of 32 inner nodes starting at the root, the two
// children tested in order (left, then right) and the right one popped first; an inner child that meets a
// full stack ends the whole query (the pairs found so far stay), and so does the 100001st popped node.
// Both early exits are reported through `capped`.  EE keeps the reference's eid < adj filter.
template <bool EE>
__global__ void __launch_bounds__(128) k_query_ref(const float4* __restrict__ wide, const float4* __restrict__ x0,
                                                   const float4* __restrict__ x1, const uint2* __restrict__ edges,
                                                   uint32_t n_queries, const float* __restrict__ dhat,
                                                   const float* __restrict__ thickness, float uniform_r,
                                                   uint2* __restrict__ pairs, uint32_t capacity, uint32_t* d_count,
                                                   uint32_t* capped, const uint32_t* __restrict__ maxdepth)
{
    if (__ldg(maxdepth) < kRefStack) return;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n_queries; q += gridDim.x * blockDim.x) {
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
            // per-vertex thickness + d_hat, or one radius for every query (the once-per-pair EE form's
            // callers: thickness 0 and one d_hat)
            const float dh = dhat ? __ldg(&dhat[v0]) : uniform_r;
            const float r = dhat ? __ldg(&thickness[v0]) + dh : uniform_r;
            box[0] = mn.x - r; box[1] = mn.y - r; box[2] = mn.z - r;
            box[3] = mx.x + r; box[4] = mx.y + r; box[5] = mx.z + r;
            if (!EE && dh < 0.0f) {  // a vertex with a negative d_hat (affine-body DOF slot) queries nothing
                box[0] = box[1] = box[2] = __int_as_float(0x7f800000);
                box[3] = box[4] = box[5] = __int_as_float(0xff800000);
            }
        }
        uint32_t stack[kRefStack];
        int sp = 0;
        uint32_t loop = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const uint32_t node = stack[--sp];
            const float4* rec = wide + 4 * node;
            bool stop = false;
            uint2 hit[2];
            uint32_t nhit = 0;
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                float4 mn, mx;
                ld_slot(rec + 2 * side, mn, mx);
                if (!stop && overlap(mn, mx, box)) {
                    const uint32_t code = __float_as_uint(mn.w);
                    if (code & 0x80000000u) {
                        const uint32_t obj = code & 0x7FFFFFFFu;
                        if (!EE || q < obj) hit[nhit++] = make_uint2(q, obj);
                    } else if (sp < (int)kRefStack) {
                        stack[sp++] = code;
                    } else {
                        stop = true;  // lbvh.cpp:344-351: the whole query ends here
                    }
                }
            }
            emit_pairs(hit, nhit, pairs, capacity, d_count);
            if (stop || ++loop > 100000u) {
                if (capped) atomicOr(capped, 1u);
                break;
            }
        }
    }
}

// EE candidates with every pair found once: the set query_template2 / fn_query_from_edges_v2 produce
// ({(a, b): a < b, query box of a overlaps leaf box of b}) when every edge's first vertex has thickness 0
// and the same d_hat r.  The query of the leaf at sorted position i visits only slots whose largest
// sorted position (`last`) exceeds i, so each pair of leaves is met from the lower position alone, with a
// culling box a few ulps wider than the query box; at a leaf the reference's own test decides, in the
// reference's direction: for q < e the query box of q against the leaf box of e, for e < q the query box
// of e (e's leaf box widened by r, exact since its thickness is 0) against the leaf box of q (q's own box).
// Pairs are written (smaller id, larger id) as the reference writes them.  Leaves of other queries are
// pruned by position, not by id, so a traversal visits about half the nodes of k_query<true>.
__global__ void __launch_bounds__(128) k_query_ee_sym(const float4* __restrict__ wide4, const uint32_t* __restrict__ sgo,
                                                      uint32_t n_leaves, const float4* __restrict__ x0,
                                                      const float4* __restrict__ x1, const uint2* __restrict__ edges,
                                                      float r, uint2* __restrict__ pairs, uint32_t capacity,
                                                      uint32_t* d_count, uint32_t* capped,
                                                      const uint32_t* __restrict__ maxdepth)
{
    if (__ldg(maxdepth) >= kRefStack) return;  // a deep tree: k_query_ref<true> (the full EE walk) instead
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_leaves; t += gridDim.x * blockDim.x) {
        const uint32_t q = __ldg(&sgo[t]);
        const uint2 ed = __ldg(&edges[q]);
        const v3 s0 = ld3(x0, ed.x), s1 = ld3(x0, ed.y), e0 = ld3(x1, ed.x), e1 = ld3(x1, ed.y);
        const v3 mn = min3(min3(s0, s1), min3(e0, e1)), mx = max3(max3(s0, s1), max3(e0, e1));
        const float4 own_mn = make_float4(mn.x, mn.y, mn.z, 0.f), own_mx = make_float4(mx.x, mx.y, mx.z, 0.f);
        const float box[6] = {mn.x - r, mn.y - r, mn.z - r, mx.x + r, mx.y + r, mx.z + r};
        float cull[6];
        {
            const float mgx = (fabsf(mn.x) + fabsf(mx.x) + r) * 9.5367431640625e-07f;  // 2^-20
            const float mgy = (fabsf(mn.y) + fabsf(mx.y) + r) * 9.5367431640625e-07f;
            const float mgz = (fabsf(mn.z) + fabsf(mx.z) + r) * 9.5367431640625e-07f;
            cull[0] = box[0] - mgx; cull[1] = box[1] - mgy; cull[2] = box[2] - mgz;
            cull[3] = box[3] + mgx; cull[4] = box[4] + mgy; cull[5] = box[5] + mgz;
        }
        uint32_t stack[kStack4];
        int sp = 0;
        uint32_t loop = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const uint32_t node = stack[--sp];
            const float4* node_rec = wide4 + 8 * node;
            float4 rec[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) ld_slot(node_rec + 2 * j, rec[2 * j], rec[2 * j + 1]);
            bool stop = false;
            uint2 hit[4];
            uint32_t nhit = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float4 cmn = rec[2 * k], cmx = rec[2 * k + 1];
                if (!stop && __float_as_uint(cmx.w) > t && overlap(cmn, cmx, cull)) {
                    const uint32_t code = __float_as_uint(cmn.w);
                    if (code & 0x80000000u) {
                        const uint32_t e = code & 0x7FFFFFFFu;
                        if (q < e) {
                            if (overlap(cmn, cmx, box)) hit[nhit++] = make_uint2(q, e);
                        } else {
                            const float qe[6] = {cmn.x - r, cmn.y - r, cmn.z - r, cmx.x + r, cmx.y + r, cmx.z + r};
                            if (overlap(own_mn, own_mx, qe)) hit[nhit++] = make_uint2(e, q);
                        }
                    } else if (sp < kStack4) {
                        stack[sp++] = code;
                    } else {
                        stop = true;
                    }
                }
            }
            emit_pairs(hit, nhit, pairs, capacity, d_count);
            if (stop || ++loop > 100000u) {
                if (capped) atomicOr(capped, 1u);
                break;
            }
        }
    }
}

// Candidate filter: the pairs of `in` whose boxes overlap at positions x (static boxes, the
// query inflated by thickness + d_hat of its first vertex, the leaf by the thickness of its
// element's first vertex, strict test), i.e. exactly what query_template2 reports at x when no
// early exit happens.  Used when `in` is a superset (the swept-box list of the same tree).
template <bool EE>
__global__ void __launch_bounds__(256) k_filter(const uint2* __restrict__ in, const uint32_t* __restrict__ in_count,
                                                uint32_t in_cap, const float4* __restrict__ x,
                                                const uint32_t* __restrict__ elems, const float* __restrict__ dhat,
                                                const float* __restrict__ thickness, uint2* __restrict__ out,
                                                uint32_t out_cap, uint32_t* out_count, const uint8_t* __restrict__ skip)
{
    uint32_t n = *in_count;
    n = n < in_cap ? n : in_cap;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n_round = (n + stride - 1) / stride * stride;  // whole warps stay in the loop for the ballot
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += stride) {
        bool keep = false;
        uint2 pr = make_uint2(0, 0);
        if (i < n) {
            pr = __ldg(&in[i]);
            v3 qa;
            uint32_t v0;
            if (EE) {
                const uint2 ed = __ldg(reinterpret_cast<const uint2*>(elems) + pr.x);
                const v3 s0 = ld3(x, ed.x), s1 = ld3(x, ed.y);
                const v3 mn = min3(min3(s0, s1), min3(s0, s1)), mx = max3(max3(s0, s1), max3(s0, s1));
                v0 = ed.x;
                const float r = __ldg(&thickness[v0]) + __ldg(&dhat[v0]);
                const float q[6] = {mn.x - r, mn.y - r, mn.z - r, mx.x + r, mx.y + r, mx.z + r};
                v3 lm, lx;
                leaf_box(LCS_TREE_EDGE, pr.y, thickness, x, x, elems, lm, lx);
                keep = overlap(make_float4(lm.x, lm.y, lm.z, 0.f), make_float4(lx.x, lx.y, lx.z, 0.f), q) &&
                       !(skip && skip[v0]);
            } else {
                qa = ld3(x, pr.x);
                const v3 mn = min3(qa, qa), mx = max3(qa, qa);
                v0 = pr.x;
                const float r = __ldg(&thickness[v0]) + __ldg(&dhat[v0]);
                const float q[6] = {mn.x - r, mn.y - r, mn.z - r, mx.x + r, mx.y + r, mx.z + r};
                v3 lm, lx;
                leaf_box(LCS_TREE_FACE, pr.y, thickness, x, x, elems, lm, lx);
                keep = overlap(make_float4(lm.x, lm.y, lm.z, 0.f), make_float4(lx.x, lx.y, lx.z, 0.f), q) &&
                       !(skip && skip[v0]);
            }
        }
        const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, keep);
        uint32_t base = 0;
        if (lane_id() == 0 && ballot) base = atomicAdd(out_count, __popc(ballot));
        base = __shfl_sync(0xFFFFFFFFu, base, 0) + __popc(ballot & ((1u << lane_id()) - 1u));
        if (keep && base < out_cap) out[base] = pr;
    }
}

__global__ void k_export(const lcs_bvh h_in, uint32_t* __restrict__ object_idx, uint64_t* __restrict__ morton,
                         float* __restrict__ node_aabb)
{
    const uint32_t n = h_in.n, ni = h_in.ni, nn = 2 * n - 1;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
        if (object_idx) object_idx[k] = k >= ni ? h_in.sgo[k - ni] : kInvalid;
        if (morton && k < n) morton[k] = ((uint64_t)h_in.m30[k] << 32) | k;
        if (node_aabb) {
            float4 mn, mx;
            if (n == 1) {
                mn = h_in.wide[0];
                mx = h_in.wide[1];
            } else if (k == 0) {
                float4 a0 = h_in.wide[0], a1 = h_in.wide[1], b0 = h_in.wide[2], b1 = h_in.wide[3];
                mn = make_float4(fmn(a0.x, b0.x), fmn(a0.y, b0.y), fmn(a0.z, b0.z), 0.0f);
                mx = make_float4(fmx(a1.x, b1.x), fmx(a1.y, b1.y), fmx(a1.z, b1.z), 0.0f);
            } else {
                uint32_t s = h_in.slot[k];
                mn = h_in.wide[4 * (s >> 1) + 2 * (s & 1u)];
                mx = h_in.wide[4 * (s >> 1) + 2 * (s & 1u) + 1];
            }
            float* o = node_aabb + 8 * (size_t)k;
            o[0] = mn.x; o[1] = mn.y; o[2] = mn.z; o[3] = 0.0f;
            o[4] = mx.x; o[5] = mx.y; o[6] = mx.z; o[7] = 0.0f;
        }
    }
}

template <typename T>
cudaError_t alloc(T*& p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (count ? count : 1));
}

}  // namespace

extern "C" int lcs_bvh_create(int kind, uint32_t n_leaves, lcs_bvh** out)
{
    if (!out || kind < LCS_TREE_VERT || kind > LCS_TREE_FACE) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_create: bad argument");
    lcs_bvh* h = new (std::nothrow) lcs_bvh();
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_create: out of host memory");
    h->kind = kind;
    h->n = n_leaves;
    h->ni = n_leaves ? n_leaves - 1 : 0;
    h->nb = (n_leaves + 255) / 256;
    const size_t nn = n_leaves ? 2 * (size_t)n_leaves - 1 : 1;
    const size_t nw = h->ni ? h->ni : 1;
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(alloc(h->centers, n_leaves));
    A(alloc(h->block_aabb, 6 * (size_t)(h->nb ? h->nb : 1)));
    A(alloc(h->gaabb, 6));
    A(alloc(h->m30, n_leaves));
    A(alloc(h->keys, n_leaves));
    A(alloc(h->keys_alt, n_leaves));
    A(alloc(h->vals, n_leaves));
    A(alloc(h->vals_alt, n_leaves));
    A(alloc(h->hist, rs::hist_words(n_leaves)));
    A(alloc(h->ms64, n_leaves));
    A(alloc(h->parent, nn));
    A(alloc(h->children, nn));
    A(alloc(h->slot, nn));
    A(alloc(h->wide, 4 * nw));
    A(alloc(h->wide4, 8 * nw));
    A(alloc(h->even, nw));
    A(alloc(h->range, nw));
    A(alloc(h->swap_diff, (size_t)n_leaves + 1));
    A(alloc(h->swap_cov, (size_t)n_leaves + 1));
    A(alloc(h->scan_tmp, scan::tmp_words(n_leaves + 1)));
    A(alloc(h->n_plus_1, 1));
    A(alloc(h->leaf_at, n_leaves));
    A(alloc(h->node_at, nw));
    A(alloc(h->order_range, nw));
    A(alloc(h->spans, nw));
    A(alloc(h->span_count, 1));
    const size_t chunks = (n_leaves + kRefitChunk - 1) / kRefitChunk;  // every chunk writes all its segments
    A(alloc(h->seg_box, 2 * chunks * kRefitSegs));
    A(alloc(h->chunk_box, 2 * chunks));
    A(alloc(h->healthy, 1));
    A(alloc(h->maxdepth, 1));
    if (e == cudaSuccess) e = cudaMemset(h->maxdepth, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(h->span_count, 0, sizeof(uint32_t));
    const uint32_t np1 = n_leaves + 1;
    if (e == cudaSuccess) e = cudaMemcpy(h->n_plus_1, &np1, sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->wide, 0, sizeof(float4) * 4 * nw);
    if (e == cudaSuccess) e = cudaMemset(h->wide4, 0, sizeof(float4) * 8 * nw);
    if (e == cudaSuccess) e = cudaMemset(h->even, 1, nw);
    if (e == cudaSuccess) e = cudaMemset(h->slot, 0xFF, sizeof(uint32_t) * nn);
    if (e != cudaSuccess) {
        lcs_bvh_destroy(h);
        return lcs_fail(LCS_ERR_CUDA, "lcs_bvh_create: cudaMalloc failed");
    }
    h->sgo = h->vals;
    h->m30_sorted = h->keys;
    *out = h;
    return LCS_OK;
}

extern "C" int lcs_bvh_destroy(lcs_bvh* h)
{
    if (!h) return LCS_OK;
    void* ptrs[] = {h->centers, h->block_aabb, h->gaabb, h->m30, h->keys, h->keys_alt, h->vals, h->vals_alt,
                    h->hist, h->ms64, h->parent, h->children, h->slot, h->wide, h->wide4, h->even, h->range,
                    h->swap_diff, h->swap_cov, h->scan_tmp, h->n_plus_1, h->leaf_at, h->node_at,
                    h->order_range, h->spans, h->span_count, h->seg_box, h->chunk_box, h->healthy, h->maxdepth};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete h;
    return LCS_OK;
}

extern "C" uint32_t lcs_bvh_num_leaves(const lcs_bvh* h) { return h ? h->n : 0; }

extern "C" int lcs_bvh_reduce_aabb(lcs_bvh* h, const float* x, const uint32_t* elems, uint32_t n_verts,
                                   lcs_stream stream)
{
    if (!h || !x || (h->kind != LCS_TREE_VERT && !elems) || n_verts == 0)
        return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_reduce_aabb: bad argument");
    if (h->kind == LCS_TREE_VERT && n_verts > 256u * 256u)
        return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_reduce_aabb: vertex tree over 65536 vertices (lbvh.cpp:941-945)");
    if (h->n == 0) return LCS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    k_reduce_pass1<<<h->nb, 256, 0, s>>>(h->kind, reinterpret_cast<const float4*>(x), elems, h->n, h->centers,
                                         h->block_aabb);
    lcs_count_launch();
    uint32_t nb_verts = (n_verts + 255) / 256;
    uint32_t cover = nb_verts < h->nb ? nb_verts : h->nb;
    k_reduce_pass2<<<1, 256, 0, s>>>(h->block_aabb, cover, h->gaabb);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

// the refit's union-order tables of a freshly built topology (k_eorder)
static cudaError_t union_order(lcs_bvh* h, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(h->span_count, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    scan::exclusive_u32(h->swap_diff, h->swap_cov, h->n_plus_1, h->n + 1, h->scan_tmp, s);
    k_eorder<<<grid_for((uint64_t)h->n + h->ni, 256), 256, 0, s>>>(h->n, h->parent, h->children, h->range,
                                                                   h->swap_cov, h->leaf_at, h->node_at,
                                                                   h->order_range, h->spans, h->span_count);
    lcs_count_launch();
    return cudaGetLastError();
}

extern "C" int lcs_bvh_construct(lcs_bvh* h, lcs_stream stream)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_construct: null handle");
    if (h->n == 0) return LCS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int g = grid_for(h->n, 256);
    k_mortons<<<g, 256, 0, s>>>(h->centers, h->gaabb, h->n, h->m30, h->keys, h->vals);
    lcs_count_launch();
    bool alt = rs::sort_pairs<uint32_t>(h->keys, h->vals, h->keys_alt, h->vals_alt, nullptr, h->n, h->n, 0, 30,
                                        h->hist, s);
    h->m30_sorted = alt ? h->keys_alt : h->keys;
    h->sgo = alt ? h->vals_alt : h->vals;
    k_apply_sorted<<<g, 256, 0, s>>>(h->m30_sorted, h->sgo, h->n, h->ms64, h->children, h->parent, h->healthy);
    lcs_count_launch();
    if (h->ni > 0) {
        const int gi = grid_for(h->ni, 256);
        LCS_CUDA_TRY(cudaMemsetAsync(h->swap_diff, 0, sizeof(uint32_t) * ((size_t)h->n + 1), s));
        k_build_inner<<<gi, 256, 0, s>>>(h->ms64, h->sgo, h->n, h->parent, h->children, h->slot, h->wide,
                                         h->maxdepth, h->range, h->swap_diff);
        lcs_count_launch();
        k_check<<<gi, 256, 0, s>>>(h->children, h->parent, h->ni, h->healthy);
        lcs_count_launch();
        k_depth_parity<<<gi, 256, 0, s>>>(h->parent, h->ni, h->even, h->maxdepth);
        lcs_count_launch();
        LCS_CUDA_TRY(union_order(h, s));
    } else {
        cudaMemcpyAsync(h->slot, &kInvalid, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    }
    LCS_LAUNCH_CHECK();
    h->built = true;
    return LCS_OK;
}

int lcs_bvh_construct_host_sort(lcs_bvh* h, lcs_stream stream)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_construct_host_sort: null handle");
    if (h->n == 0) return LCS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    k_mortons<<<grid_for(h->n, 256), 256, 0, s>>>(h->centers, h->gaabb, h->n, h->m30, h->keys, h->vals);
    lcs_count_launch();
    std::vector<uint32_t> m(h->n), idx(h->n);
    LCS_CUDA_TRY(cudaMemcpyAsync(m.data(), h->m30, 4 * (size_t)h->n, cudaMemcpyDeviceToHost, s));
    LCS_CUDA_TRY(cudaStreamSynchronize(s));
    for (uint32_t i = 0; i < h->n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
        const uint64_t ka = ((uint64_t)m[a] << 32) | a, kb = ((uint64_t)m[b] << 32) | b;
        return ka < kb;
    });
    std::vector<uint32_t> ms(h->n);
    for (uint32_t i = 0; i < h->n; ++i) ms[i] = m[idx[i]];
    h->m30_sorted = h->keys;
    h->sgo = h->vals;
    LCS_CUDA_TRY(cudaMemcpyAsync(h->m30_sorted, ms.data(), 4 * (size_t)h->n, cudaMemcpyHostToDevice, s));
    LCS_CUDA_TRY(cudaMemcpyAsync(h->sgo, idx.data(), 4 * (size_t)h->n, cudaMemcpyHostToDevice, s));
    const int g = grid_for(h->n, 256);
    k_apply_sorted<<<g, 256, 0, s>>>(h->m30_sorted, h->sgo, h->n, h->ms64, h->children, h->parent, h->healthy);
    lcs_count_launch();
    if (h->ni > 0) {
        const int gi = grid_for(h->ni, 256);
        LCS_CUDA_TRY(cudaMemsetAsync(h->swap_diff, 0, sizeof(uint32_t) * ((size_t)h->n + 1), s));
        k_build_inner<<<gi, 256, 0, s>>>(h->ms64, h->sgo, h->n, h->parent, h->children, h->slot, h->wide,
                                         h->maxdepth, h->range, h->swap_diff);
        lcs_count_launch();
        k_check<<<gi, 256, 0, s>>>(h->children, h->parent, h->ni, h->healthy);
        lcs_count_launch();
        k_depth_parity<<<gi, 256, 0, s>>>(h->parent, h->ni, h->even, h->maxdepth);
        lcs_count_launch();
        LCS_CUDA_TRY(union_order(h, s));
    }
    LCS_CUDA_TRY(cudaStreamSynchronize(s));  // host buffers go out of scope
    LCS_LAUNCH_CHECK();
    h->built = true;
    return LCS_OK;
}

static int leaves_refit(lcs_bvh* h, const float* thickness, const float* x0, const float* x1, const uint32_t* elems,
                        int write_leaf, int climb, lcs_stream stream)
{
    if (!h || (write_leaf && (!thickness || !x0 || !x1 || (h->kind != LCS_TREE_VERT && !elems))))
        return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_update/refit: bad argument");
    if (h->n == 0) return LCS_OK;
    // the slots and refit tables are written by the build: before it they hold no valid indices
    if (!h->built) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_update/refit: the tree has not been constructed");
    cudaStream_t s = (cudaStream_t)stream;
    const float4* px0 = reinterpret_cast<const float4*>(x0);
    const float4* px1 = reinterpret_cast<const float4*>(x1);
    if (climb && h->n > 1) {
        const uint32_t chunks = (h->n + kRefitChunk - 1) / kRefitChunk;
        k_refit_chunks<<<chunks, kRefitChunk, 0, s>>>(h->kind, h->n, h->sgo, h->slot, h->leaf_at, h->node_at,
                                                      h->order_range, h->even, thickness,
                                                      px0, px1, elems, write_leaf, h->wide, h->wide4, h->seg_box,
                                                      h->chunk_box);
        lcs_count_launch();
        if (chunks > 1) {
            // one warp per crossing node in one round: about ten crossing nodes per chunk on the tube's trees,
            // 8 warps per block, at most the 5 blocks per SM that 44 registers a thread allow
            const uint32_t span_blocks = 2 * chunks < 5u * kNumSMs ? 2 * chunks : 5u * kNumSMs;
            k_refit_spans<<<span_blocks, 256, 0, s>>>(h->n, h->spans, h->span_count, h->order_range, h->leaf_at,
                                                      h->slot,
                                                            h->seg_box, h->chunk_box, h->wide);
            lcs_count_launch();
            k_refit_span_records<<<kNumSMs, 256, 0, s>>>(h->spans, h->span_count, h->even, h->wide,
                                                               h->wide4);
            lcs_count_launch();
        }
    } else if (write_leaf) {
        k_leaves<<<grid_for(h->n, 256), 256, 0, s>>>(h->kind, h->n, h->sgo, h->slot, thickness, px0, px1, elems,
                                                     h->wide, h->wide4);
        lcs_count_launch();
    }
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_bvh_update_leaves(lcs_bvh* h, const float* thickness, const float* x0, const float* x1,
                                     const uint32_t* elems, lcs_stream stream)
{
    return leaves_refit(h, thickness, x0, x1, elems, 1, 0, stream);
}

extern "C" int lcs_bvh_refit(lcs_bvh* h, lcs_stream stream)
{
    return leaves_refit(h, nullptr, nullptr, nullptr, nullptr, 0, 1, stream);
}

extern "C" int lcs_bvh_update_refit(lcs_bvh* h, const float* thickness, const float* x0, const float* x1,
                                    const uint32_t* elems, lcs_stream stream)
{
    return leaves_refit(h, thickness, x0, x1, elems, 1, 1, stream);
}

extern "C" int lcs_bvh_query_vf(const lcs_bvh* t, const float* x0, const float* x1, uint32_t n_verts,
                                const float* d_hat, const float* thickness, uint32_t* pairs, uint32_t capacity,
                                uint32_t* d_count, lcs_stream stream)
{
    return lcs_bvh_query_vf_capped(t, x0, x1, n_verts, d_hat, thickness, pairs, capacity, d_count, nullptr, stream);
}

int lcs_bvh_query_vf_capped(const lcs_bvh* t, const float* x0, const float* x1, uint32_t n_verts, const float* d_hat,
                            const float* thickness, uint32_t* pairs, uint32_t capacity, uint32_t* d_count,
                            uint32_t* capped, lcs_stream stream)
{
    if (!t || t->kind != LCS_TREE_FACE || !x0 || !x1 || !d_hat || !thickness || !d_count || (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_query_vf: bad argument (needs a face tree)");
    if (t->n == 0 || n_verts == 0) return LCS_OK;
    if (!t->built) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_query_vf: the tree has not been constructed");
    k_query<false><<<grid_for(n_verts, 128, 16), 128, 0, (cudaStream_t)stream>>>(
        t->wide4, t->n, reinterpret_cast<const float4*>(x0), reinterpret_cast<const float4*>(x1), nullptr, n_verts,
        d_hat, thickness, reinterpret_cast<uint2*>(pairs), capacity, d_count, nullptr, capped, t->maxdepth);
    lcs_count_launch();
    if (t->ni > 0) {
        k_query_ref<false><<<grid_for(n_verts, 128, 16), 128, 0, (cudaStream_t)stream>>>(
            t->wide, reinterpret_cast<const float4*>(x0), reinterpret_cast<const float4*>(x1), nullptr, n_verts, d_hat,
            thickness, 0.0f, reinterpret_cast<uint2*>(pairs), capacity, d_count, capped, t->maxdepth);
        lcs_count_launch();
    }
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_bvh_query_ee(const lcs_bvh* t, const float* x0, const float* x1, const uint32_t* edges,
                                uint32_t n_edges, const float* d_hat, const float* thickness, uint32_t* pairs,
                                uint32_t capacity, uint32_t* d_count, lcs_stream stream)
{
    return lcs_bvh_query_ee_capped(t, x0, x1, edges, n_edges, d_hat, thickness, pairs, capacity, d_count, nullptr,
                                   stream);
}

int lcs_bvh_query_ee_capped(const lcs_bvh* t, const float* x0, const float* x1, const uint32_t* edges, uint32_t n_edges,
                            const float* d_hat, const float* thickness, uint32_t* pairs, uint32_t capacity,
                            uint32_t* d_count, uint32_t* capped, lcs_stream stream)
{
    if (!t || t->kind != LCS_TREE_EDGE || !x0 || !x1 || !edges || !d_hat || !thickness || !d_count ||
        (capacity && !pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_query_ee: bad argument (needs an edge tree)");
    if (t->n == 0 || n_edges == 0) return LCS_OK;
    if (!t->built) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_query_ee: the tree has not been constructed");
    k_query<true><<<grid_for(n_edges, 128, 16), 128, 0, (cudaStream_t)stream>>>(
        t->wide4, t->n, reinterpret_cast<const float4*>(x0), reinterpret_cast<const float4*>(x1),
        reinterpret_cast<const uint2*>(edges), n_edges, d_hat, thickness, reinterpret_cast<uint2*>(pairs), capacity,
        d_count, n_edges == t->n ? t->sgo : nullptr, capped, t->maxdepth);
    lcs_count_launch();
    if (t->ni > 0) {
        k_query_ref<true><<<grid_for(n_edges, 128, 16), 128, 0, (cudaStream_t)stream>>>(
            t->wide, reinterpret_cast<const float4*>(x0), reinterpret_cast<const float4*>(x1),
            reinterpret_cast<const uint2*>(edges), n_edges, d_hat, thickness, 0.0f, reinterpret_cast<uint2*>(pairs),
            capacity, d_count, capped, t->maxdepth);
        lcs_count_launch();
    }
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_bvh_query_ee_sym(const lcs_bvh* t, const float* x0, const float* x1, const uint32_t* edges,
                                    float d_hat, uint32_t* pairs, uint32_t capacity, uint32_t* d_count,
                                    lcs_stream stream)
{
    return lcs_bvh_query_ee_sym_capped(t, x0, x1, edges, d_hat, pairs, capacity, d_count, nullptr, stream);
}

int lcs_bvh_query_ee_sym_capped(const lcs_bvh* t, const float* x0, const float* x1, const uint32_t* edges,
                                float d_hat, uint32_t* pairs, uint32_t capacity, uint32_t* d_count, uint32_t* capped,
                                lcs_stream stream)
{
    if (!t || t->kind != LCS_TREE_EDGE || !x0 || !x1 || !edges || !d_count || (capacity && !pairs) ||
        !(d_hat >= 0.0f))
        return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_query_ee_sym: bad argument (needs an edge tree, d_hat >= 0)");
    if (t->n == 0) return LCS_OK;
    if (!t->built) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_query_ee_sym: the tree has not been constructed");
    k_query_ee_sym<<<grid_for(t->n, 128, 16), 128, 0, (cudaStream_t)stream>>>(
        t->wide4, t->sgo, t->n, reinterpret_cast<const float4*>(x0), reinterpret_cast<const float4*>(x1),
        reinterpret_cast<const uint2*>(edges), d_hat, reinterpret_cast<uint2*>(pairs), capacity, d_count, capped,
        t->maxdepth);
    lcs_count_launch();
    if (t->ni > 0) {  // a deep tree: the reference's full EE walk (its early exits break the symmetry)
        k_query_ref<true><<<grid_for(t->n, 128, 16), 128, 0, (cudaStream_t)stream>>>(
            t->wide, reinterpret_cast<const float4*>(x0), reinterpret_cast<const float4*>(x1),
            reinterpret_cast<const uint2*>(edges), t->n, nullptr, nullptr, d_hat, reinterpret_cast<uint2*>(pairs),
            capacity, d_count, capped, t->maxdepth);
        lcs_count_launch();
    }
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_bvh_health(lcs_bvh* h, int* healthy, lcs_stream stream)
{
    if (!h || !healthy) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_health: bad argument");
    if (h->n == 0) { *healthy = 1; return LCS_OK; }
    uint32_t v = 0;
    LCS_CUDA_TRY(cudaMemcpyAsync(&v, h->healthy, sizeof(uint32_t), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    LCS_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    *healthy = (int)v;
    return LCS_OK;
}

// fn_check_construction (lbvh.cpp:598-611) on the tree as it is now
extern "C" int lcs_bvh_check_construction(lcs_bvh* h, lcs_stream stream)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_check_construction: null handle");
    if (h->ni == 0) return LCS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    k_set_healthy<<<1, 1, 0, s>>>(h->healthy);
    lcs_count_launch();
    k_check<<<grid_for(h->ni, 256), 256, 0, s>>>(h->children, h->parent, h->ni, h->healthy);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_bvh_data(const lcs_bvh* h, lcs_bvh_data_view* out)
{
    if (!h || !out) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_data: null argument");
    out->n_leaves = h->n;
    out->parent = h->parent;
    out->children = reinterpret_cast<uint32_t*>(h->children);
    out->morton_sorted = h->ms64;
    out->sorted_get_original = h->sgo;
    out->is_healthy = h->healthy;
    return LCS_OK;
}

extern "C" int lcs_bvh_export(const lcs_bvh* h, uint32_t* parent, uint32_t* children, uint32_t* object_idx,
                              uint64_t* morton, uint64_t* morton_sorted, uint32_t* sorted_get_original,
                              float* node_aabb, float* global_aabb6, lcs_stream stream)
{
    if (!h) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_export: null handle");
    if (h->n == 0) return LCS_OK;
    if (!h->built) return lcs_fail(LCS_ERR_INVALID, "lcs_bvh_export: the tree has not been constructed");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nn = 2 * (size_t)h->n - 1;
    if (parent) LCS_CUDA_TRY(cudaMemcpyAsync(parent, h->parent, 4 * nn, cudaMemcpyDeviceToDevice, s));
    if (children) LCS_CUDA_TRY(cudaMemcpyAsync(children, h->children, 8 * nn, cudaMemcpyDeviceToDevice, s));
    if (morton_sorted) LCS_CUDA_TRY(cudaMemcpyAsync(morton_sorted, h->ms64, 8 * (size_t)h->n, cudaMemcpyDeviceToDevice, s));
    if (sorted_get_original) LCS_CUDA_TRY(cudaMemcpyAsync(sorted_get_original, h->sgo, 4 * (size_t)h->n, cudaMemcpyDeviceToDevice, s));
    if (global_aabb6) LCS_CUDA_TRY(cudaMemcpyAsync(global_aabb6, h->gaabb, 24, cudaMemcpyDeviceToDevice, s));
    if (object_idx || morton || node_aabb) {
        k_export<<<grid_for(nn, 256), 256, 0, s>>>(*h, object_idx, morton, node_aabb);
        lcs_count_launch();
    }
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

int lcs_candidates_filter_masked(int is_ee, const uint32_t* in_pairs, const uint32_t* in_count, uint32_t in_capacity,
                                 const float* x, const uint32_t* elems, const float* d_hat, const float* thickness,
                                 uint32_t* out_pairs, uint32_t out_capacity, uint32_t* out_count, lcs_stream stream,
                                 const uint8_t* skip)
{
    if (!in_count || !x || !elems || !d_hat || !thickness || !out_count || (in_capacity && !in_pairs) ||
        (out_capacity && !out_pairs))
        return lcs_fail(LCS_ERR_INVALID, "lcs_candidates_filter: bad argument");
    if (in_capacity == 0) return LCS_OK;
    auto kern = is_ee ? k_filter<true> : k_filter<false>;
    kern<<<grid_for(in_capacity, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const uint2*>(in_pairs), in_count, in_capacity, reinterpret_cast<const float4*>(x), elems,
        d_hat, thickness, reinterpret_cast<uint2*>(out_pairs), out_capacity, out_count, skip);
    lcs_count_launch();
    LCS_LAUNCH_CHECK();
    return LCS_OK;
}

extern "C" int lcs_candidates_filter(int is_ee, const uint32_t* in_pairs, const uint32_t* in_count, uint32_t in_capacity,
                                     const float* x, const uint32_t* elems, const float* d_hat, const float* thickness,
                                     uint32_t* out_pairs, uint32_t out_capacity, uint32_t* out_count, lcs_stream stream)
{
    return lcs_candidates_filter_masked(is_ee, in_pairs, in_count, in_capacity, x, elems, d_hat, thickness, out_pairs,
                                        out_capacity, out_count, stream, nullptr);
}

