/*
 * lcs_oracle.c -- CPU restatement (C11 + OpenMP) of the contact-and-solve path of
 * LuisaComputeSimulator.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, and the
 * timed CPU baseline of bench.py.  The product never links it.
 *
 * Every function names the reference file:line it restates.  Device semantics are followed
 * (the LuisaCompute shaders), including their quirks, because the sorted candidate sets and
 * the BVH topology must match bit for bit.  See lcs_oracle.h for layouts and pin status.
 */
#include "lcs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)

#define T float
#define SFX _f
#define FMA fmaf
#include "lcs_oracle_geom.inc"
#undef T
#undef SFX
#undef FMA

#define T double
#define SFX _d
#define FMA fma
#include "lcs_oracle_geom.inc"
#undef T
#undef SFX
#undef FMA

static inline v3_f ld3(const float* x4, uint32_t i)
{
    return mk_f(x4[4 * (size_t)i + 0], x4[4 * (size_t)i + 1], x4[4 * (size_t)i + 2]);
}
static inline v3_f ldp(const float* p) { return mk_f(p[0], p[1], p[2]); }
static inline float fminf_(float a, float b) { return a < b ? a : b; }
static inline float fmaxf_(float a, float b) { return a > b ? a : b; }

/* =========================================================================================
 * LBVH  (Solver/CollisionDetector/lbvh.cpp)
 * ========================================================================================= */

/* lbvh.cpp:84-91 */
static inline uint32_t expand_bits(uint32_t v)
{
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    return (v | (v << 2)) & 0x09249249u;
}

/* lbvh.cpp:112-124: 10 bits per axis, clamp to [0, 1023], truncate, interleave x<<2|y<<1|z */
static inline uint32_t morton32(float px, float py, float pz)
{
    float x = px * 1024.0f, y = py * 1024.0f, z = pz * 1024.0f;
    x = fminf_(fmaxf_(x, 0.0f), 1023.0f);
    y = fminf_(fmaxf_(y, 0.0f), 1023.0f);
    z = fminf_(fmaxf_(z, 0.0f), 1023.0f);
    uint32_t xx = expand_bits((uint32_t)x), yy = expand_bits((uint32_t)y), zz = expand_bits((uint32_t)z);
    return (xx << 2) | (yy << 1) | zz;
}

/* LBVH::unit_test inputs, lbvh.cpp:898-910: leaf i at (i/10, i/10, i/10) */
void orc_morton_codes_unit(uint32_t n, uint32_t* m32, uint64_t* m64)
{
    for (uint32_t i = 0; i < n; ++i) {
        float pos = (float)i / 10.0f;
        m32[i] = morton32(pos, pos, pos);
        m64[i] = ((uint64_t)m32[i] << 32) | (uint64_t)i;
    }
}

static inline void elem_box(int kind, const float* x, const uint32_t* elems, uint32_t e,
                            v3_f* mn, v3_f* mx, v3_f* center)
{
    if (kind == ORC_TREE_VERT) {
        v3_f p = ld3(x, e);
        *mn = p; *mx = p; *center = p;
    } else if (kind == ORC_TREE_EDGE) {
        v3_f p0 = ld3(x, elems[2 * (size_t)e]), p1 = ld3(x, elems[2 * (size_t)e + 1]);
        *mn = mk_f(fminf_(p0.x, p1.x), fminf_(p0.y, p1.y), fminf_(p0.z, p1.z));
        *mx = mk_f(fmaxf_(p0.x, p1.x), fmaxf_(p0.y, p1.y), fmaxf_(p0.z, p1.z));
        *center = scl_f(0.5f, add_f(p0, p1)); /* lbvh.cpp:468 */
    } else {
        v3_f p0 = ld3(x, elems[4 * (size_t)e]), p1 = ld3(x, elems[4 * (size_t)e + 1]),
             p2 = ld3(x, elems[4 * (size_t)e + 2]);
        *mn = mk_f(fminf_(p0.x, fminf_(p1.x, p2.x)), fminf_(p0.y, fminf_(p1.y, p2.y)),
                   fminf_(p0.z, fminf_(p1.z, p2.z)));
        *mx = mk_f(fmaxf_(p0.x, fmaxf_(p1.x, p2.x)), fmaxf_(p0.y, fmaxf_(p1.y, p2.y)),
                   fmaxf_(p0.z, fmaxf_(p1.z, p2.z)));
        *center = scl_f(0.333333f, add_f(add_f(p0, p1), p2)); /* lbvh.cpp:488 */
    }
}

/*
 * Global AABB for Morton normalisation: lbvh.cpp:368-491 (first pass, one partial per 256
 * elements) and lbvh.cpp:939-973 (second pass).  Quirk kept on purpose: the second pass is
 * dispatched over ceil(n_verts / 256) partials for every tree kind, so the edge and face trees
 * only see elements [0, 256 * ceil(n_verts / 256)).  Partials beyond the ones the first pass
 * wrote are never read here (the reference would read past its buffer there).
 */
void orc_lbvh_reduce_aabb(int kind, const float* x, const uint32_t* elems, uint32_t n_elems,
                          uint32_t n_verts, float* gmin3, float* gmax3, float* centers4)
{
    uint32_t nb_elems = (n_elems + 255u) / 256u;
    uint32_t nb_verts = (n_verts + 255u) / 256u;
    uint32_t nb = nb_verts < nb_elems ? nb_verts : nb_elems;
    uint64_t covered = (uint64_t)nb * 256u;
    if (covered > n_elems) covered = n_elems;
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (uint32_t e = 0; e < n_elems; ++e) {
        v3_f a, b, c;
        elem_box(kind, x, elems, e, &a, &b, &c);
        if (centers4) {
            centers4[4 * (size_t)e + 0] = c.x;
            centers4[4 * (size_t)e + 1] = c.y;
            centers4[4 * (size_t)e + 2] = c.z;
            centers4[4 * (size_t)e + 3] = 0.0f;
        }
        if (e < covered) {
            mn[0] = fminf_(mn[0], a.x); mn[1] = fminf_(mn[1], a.y); mn[2] = fminf_(mn[2], a.z);
            mx[0] = fmaxf_(mx[0], b.x); mx[1] = fmaxf_(mx[1], b.y); mx[2] = fmaxf_(mx[2], b.z);
        }
    }
    memcpy(gmin3, mn, sizeof(mn));
    memcpy(gmax3, mx, sizeof(mx));
}

/* fn_compute_mortons, lbvh.cpp:507-523 */
void orc_lbvh_mortons(const float* centers4, uint32_t n, const float* gmin3, const float* gmax3,
                      uint64_t* morton)
{
    float inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0f / fmaxf_(gmax3[k] - gmin3[k], 1e-6f);
    for (uint32_t i = 0; i < n; ++i) {
        float px = (centers4[4 * (size_t)i + 0] - gmin3[0]) * inv[0];
        float py = (centers4[4 * (size_t)i + 1] - gmin3[1]) * inv[1];
        float pz = (centers4[4 * (size_t)i + 2] - gmin3[2]) * inv[2];
        morton[i] = ((uint64_t)morton32(px, py, pz) << 32) | (uint64_t)i;
    }
}

static int cmp_u64(const void* a, const void* b)
{
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* construct_tree's host sort (lbvh.cpp:983-993): leaf ids ordered by morton64 (keys unique) */
void orc_lbvh_sort(const uint64_t* morton, uint32_t n, uint32_t* sorted_get_original,
                   uint64_t* morton_sorted)
{
    memcpy(morton_sorted, morton, sizeof(uint64_t) * n);
    qsort(morton_sorted, n, sizeof(uint64_t), cmp_u64);
    for (uint32_t i = 0; i < n; ++i) sorted_get_original[i] = (uint32_t)(morton_sorted[i] & 0xFFFFFFFFu);
}

static inline int clz64(uint64_t x) { return x == 0 ? 64 : __builtin_clzll(x); }

/* cp_i_j, lbvh.cpp:188-193 */
static inline int cp_ij(uint64_t mi, int j, const uint64_t* ms, uint32_t n)
{
    return (j >= 0 && (uint32_t)j < n) ? clz64(mi ^ ms[j]) : -1;
}

/* determineRange, lbvh.cpp:204-244 */
static void determine_range(int i, const uint64_t* ms, uint32_t n, int* ri, int* rj)
{
    uint64_t mi = ms[i];
    int cp_left = clz64(mi ^ ms[i - 1]);
    int cp_right = clz64(mi ^ ms[i + 1]);
    int d = cp_left < cp_right ? 1 : -1;
    int cp_min = cp_left < cp_right ? cp_left : cp_right;
    int lmax = 2;
    while (cp_ij(mi, i + lmax * d, ms, n) > cp_min) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (cp_ij(mi, i + (l + t) * d, ms, n) > cp_min) l += t;
    *ri = i;
    *rj = i + l * d;
}

/* findSplit, lbvh.cpp:246-291 */
static int find_split(int r0, int r1, const uint64_t* ms)
{
    int i = r0, j = r1;
    if (r0 > r1) { i = r1; j = r0; }
    uint64_t mi = ms[i], mj = ms[j];
    int cp_node = clz64(mi ^ mj);
    if (mi == mj) return (i + j) >> 1;
    int t = j - i, split = i;
    for (;;) {
        t = (t + 1) >> 1;
        int ns = split + t;
        if (ns < j && clz64(mi ^ ms[ns]) > cp_node) split = ns;
        if (!(t > 1)) break;
    }
    return split;
}

/*
 * fn_build_inner_nodes, lbvh.cpp:541-596 (+ fn_reset_tree's parent[0] = -1, lbvh.cpp:493-505).
 * Children: leaf indices are num_inner + sorted position; the pair is swapped when the right
 * child is a leaf (lbvh.cpp:575-584).  Returns the health flag of fn_check_construction
 * (lbvh.cpp:598-611).  ranges2 / splits may be NULL.
 */
int orc_lbvh_build_inner(const uint64_t* ms, uint32_t n, uint32_t* parent, uint32_t* children2,
                         int32_t* ranges2, int32_t* splits)
{
    if (n == 0) return 1;
    int ni = (int)n - 1;
    parent[0] = 0xFFFFFFFFu;
    for (int nid = 0; nid < ni; ++nid) {
        int i = 0, j = ni;
        if (nid != 0) determine_range(nid, ms, n, &i, &j);
        int split = find_split(i, j, ms);
        int lo = i < j ? i : j, hi = i < j ? j : i;
        int cl = (lo == split) ? ni + split : split;
        int cr = (hi == split + 1) ? ni + split + 1 : split + 1;
        if (cr >= ni) { int t = cl; cl = cr; cr = t; }
        parent[cl] = (uint32_t)nid;
        parent[cr] = (uint32_t)nid;
        children2[2 * nid + 0] = (uint32_t)cl;
        children2[2 * nid + 1] = (uint32_t)cr;
        if (ranges2) { ranges2[2 * nid] = i; ranges2[2 * nid + 1] = j; }
        if (splits) splits[nid] = split;
    }
    int healthy = 1;
    for (int nid = 0; nid < ni; ++nid)
        if (parent[children2[2 * nid]] != (uint32_t)nid || parent[children2[2 * nid + 1]] != (uint32_t)nid)
            healthy = 0;
    return healthy;
}

/* fn_reset_tree + fn_apply_sorted + fn_build_inner_nodes + fn_check_construction */
int orc_lbvh_construct(const uint64_t* ms, const uint32_t* sorted_get_original, uint32_t n,
                       uint32_t* parent, uint32_t* children2, uint32_t* object_idx)
{
    if (n == 0) return 1;
    uint32_t ni = n - 1, nn = 2 * n - 1;
    for (uint32_t k = 0; k < nn; ++k) object_idx[k] = 0xFFFFFFFFu;
    parent[0] = 0xFFFFFFFFu;
    for (uint32_t lid = 0; lid < n; ++lid) {
        uint32_t orig = sorted_get_original[lid];
        children2[2 * (ni + lid) + 0] = orig;
        children2[2 * (ni + lid) + 1] = orig;
        object_idx[ni + lid] = orig;
    }
    return orc_lbvh_build_inner(ms, n, parent, children2, NULL, NULL);
}

/* fn_update_{vert,edge,face}_tree_leave_aabb_v2, lbvh.cpp:617-683: swept box, +-thickness of
 * the element's first vertex; node layout = 2 float4 {min.xyz, flag0} {max.xyz, flag1}. */
void orc_lbvh_update_leaves(int kind, const uint32_t* sgo, uint32_t n, const float* thickness,
                            const float* x0, const float* x1, const uint32_t* elems,
                            float* node_aabb8)
{
    if (n == 0) return;
    uint32_t ni = n - 1;
    for (uint32_t lid = 0; lid < n; ++lid) {
        uint32_t e = sgo[lid];
        v3_f mn, mx;
        float th;
        if (kind == ORC_TREE_VERT) {
            v3_f a = ld3(x0, e), b = ld3(x1, e);
            mn = mk_f(fminf_(a.x, b.x), fminf_(a.y, b.y), fminf_(a.z, b.z));
            mx = mk_f(fmaxf_(a.x, b.x), fmaxf_(a.y, b.y), fmaxf_(a.z, b.z));
            th = thickness[e];
        } else if (kind == ORC_TREE_EDGE) {
            uint32_t v0 = elems[2 * (size_t)e], v1 = elems[2 * (size_t)e + 1];
            v3_f s0 = ld3(x0, v0), s1 = ld3(x0, v1), e0 = ld3(x1, v0), e1 = ld3(x1, v1);
            /* AABB::make_aabb(p1,p2,p3,p4) = min(min(p1,p2), min(p3,p4)), aabb.h:58-62 */
            mn = mk_f(fminf_(fminf_(s0.x, s1.x), fminf_(e0.x, e1.x)), fminf_(fminf_(s0.y, s1.y), fminf_(e0.y, e1.y)),
                      fminf_(fminf_(s0.z, s1.z), fminf_(e0.z, e1.z)));
            mx = mk_f(fmaxf_(fmaxf_(s0.x, s1.x), fmaxf_(e0.x, e1.x)), fmaxf_(fmaxf_(s0.y, s1.y), fmaxf_(e0.y, e1.y)),
                      fmaxf_(fmaxf_(s0.z, s1.z), fmaxf_(e0.z, e1.z)));
            th = thickness[v0];
        } else {
            uint32_t f0 = elems[4 * (size_t)e], f1 = elems[4 * (size_t)e + 1], f2 = elems[4 * (size_t)e + 2];
            v3_f s0 = ld3(x0, f0), s1 = ld3(x0, f1), s2 = ld3(x0, f2);
            v3_f e0 = ld3(x1, f0), e1 = ld3(x1, f1), e2 = ld3(x1, f2);
            v3_f smn = mk_f(fminf_(s0.x, fminf_(s1.x, s2.x)), fminf_(s0.y, fminf_(s1.y, s2.y)), fminf_(s0.z, fminf_(s1.z, s2.z)));
            v3_f smx = mk_f(fmaxf_(s0.x, fmaxf_(s1.x, s2.x)), fmaxf_(s0.y, fmaxf_(s1.y, s2.y)), fmaxf_(s0.z, fmaxf_(s1.z, s2.z)));
            v3_f emn = mk_f(fminf_(e0.x, fminf_(e1.x, e2.x)), fminf_(e0.y, fminf_(e1.y, e2.y)), fminf_(e0.z, fminf_(e1.z, e2.z)));
            v3_f emx = mk_f(fmaxf_(e0.x, fmaxf_(e1.x, e2.x)), fmaxf_(e0.y, fmaxf_(e1.y, e2.y)), fmaxf_(e0.z, fmaxf_(e1.z, e2.z)));
            mn = mk_f(fminf_(smn.x, emn.x), fminf_(smn.y, emn.y), fminf_(smn.z, emn.z));
            mx = mk_f(fmaxf_(smx.x, emx.x), fmaxf_(smx.y, emx.y), fmaxf_(smx.z, emx.z));
            th = thickness[f0];
        }
        float* o = node_aabb8 + 8 * (size_t)(ni + lid);
        o[0] = mn.x - th; o[1] = mn.y - th; o[2] = mn.z - th; o[3] = 0.0f;
        o[4] = mx.x + th; o[5] = mx.y + th; o[6] = mx.z + th; o[7] = 1.0f;
    }
}

/* fn_init_tree_aabb_and_flag + fn_refit_tree_aabb, lbvh.cpp:689-754: every inner node becomes
 * the union of its two children (order-independent, so a post-order walk gives the same
 * bits).  Returns 0 when the parent links do not form a tree. */
int orc_lbvh_refit(uint32_t n, const uint32_t* parent, const uint32_t* children2, float* node_aabb8)
{
    (void)parent;
    if (n <= 1) return 1;
    uint32_t ni = n - 1;
    for (uint32_t k = 0; k < ni; ++k) {
        float* o = node_aabb8 + 8 * (size_t)k;
        o[0] = o[1] = o[2] = 1e8f; o[3] = 0.0f;
        o[4] = o[5] = o[6] = -1e8f; o[7] = 0.0f;
    }
    /* iterative post-order */
    uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (size_t)n);
    uint8_t* state = (uint8_t*)calloc(ni, 1);
    int sp = 0, healthy = 1;
    size_t guard = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        if (++guard > 8u * (size_t)n) { healthy = 0; break; }
        uint32_t node = stack[sp - 1];
        if (node >= ni) { sp--; continue; }
        if (state[node] == 0) {
            state[node] = 1;
            uint32_t c0 = children2[2 * node], c1 = children2[2 * node + 1];
            if (c1 < ni) stack[sp++] = c1;
            if (c0 < ni) stack[sp++] = c0;
            continue;
        }
        sp--;
        uint32_t c0 = children2[2 * node], c1 = children2[2 * node + 1];
        const float* a = node_aabb8 + 8 * (size_t)c0;
        const float* b = node_aabb8 + 8 * (size_t)c1;
        float* o = node_aabb8 + 8 * (size_t)node;
        o[0] = fminf_(a[0], b[0]); o[1] = fminf_(a[1], b[1]); o[2] = fminf_(a[2], b[2]); o[3] = 0.0f;
        o[4] = fmaxf_(a[4], b[4]); o[5] = fmaxf_(a[5], b[5]); o[6] = fmaxf_(a[6], b[6]); o[7] = 0.0f;
    }
    free(stack);
    free(state);
    return healthy;
}

/* AABB::is_overlap_aabb with strict comparisons, aabb.h:95-100 */
static inline int overlap(const float* node, const float* q)
{
    return node[0] < q[4] && node[1] < q[5] && node[2] < q[6] && node[4] > q[0] && node[5] > q[1] &&
           node[6] > q[2];
}

/* query_template2, lbvh.cpp:293-360: stack of 32, root's own box is not tested, a full stack
 * ends the whole traversal, 100000-iteration cap.  eid_filter != 0xFFFFFFFF keeps eid < adj. */
static uint32_t query_one(const float* node_aabb8, const uint32_t* children2, const uint32_t* object_idx,
                          const float* q, uint32_t qid, uint32_t eid_filter, uint32_t* out, uint32_t cap)
{
    uint32_t stack[32];
    int sp = 0;
    uint32_t found = 0, loop = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        sp--;
        uint32_t node = stack[sp];
        int stop = 0;
        for (int ii = 0; ii < 2; ++ii) {
            uint32_t c = children2[2 * (size_t)node + ii];
            if (overlap(node_aabb8 + 8 * (size_t)c, q)) {
                uint32_t adj = object_idx[c];
                if (adj != 0xFFFFFFFFu) {
                    if (eid_filter == 0xFFFFFFFFu || eid_filter < adj) {
                        if (found < cap) { out[2 * found] = qid; out[2 * found + 1] = adj; }
                        found++;
                    }
                } else if (sp < 32) {
                    stack[sp++] = c;
                } else {
                    stop = 1;
                    break;
                }
            }
        }
        if (stop) break;
        if (++loop > 100000) break;
    }
    return found;
}

typedef struct { uint32_t* data; uint32_t n, cap; } pairbuf;

static uint32_t gather_pairs(pairbuf* bufs, int nb, uint32_t* pairs, uint32_t capacity)
{
    uint32_t total = 0;
    for (int t = 0; t < nb; ++t) {
        for (uint32_t k = 0; k < bufs[t].n; ++k) {
            if (total < capacity) {
                pairs[2 * (size_t)total] = bufs[t].data[2 * (size_t)k];
                pairs[2 * (size_t)total + 1] = bufs[t].data[2 * (size_t)k + 1];
            }
            total++;
        }
        free(bufs[t].data);
    }
    return total;
}

static void push_pairs(pairbuf* b, const uint32_t* tmp, uint32_t cnt)
{
    if (b->n + cnt > b->cap) {
        uint32_t nc = b->cap ? b->cap * 2 : 1024;
        while (nc < b->n + cnt) nc *= 2;
        b->data = (uint32_t*)realloc(b->data, sizeof(uint32_t) * 2 * (size_t)nc);
        b->cap = nc;
    }
    memcpy(b->data + 2 * (size_t)b->n, tmp, sizeof(uint32_t) * 2 * (size_t)cnt);
    b->n += cnt;
}

#ifdef _OPENMP
#include <omp.h>
#define NTHREADS omp_get_max_threads()
#define TID omp_get_thread_num()
#else
#define NTHREADS 1
#define TID 0
#endif

/* fn_query_from_verts_v2, lbvh.cpp:776-808: box = [x0, x1] +- (thickness + d_hat) of the vertex */
uint32_t orc_lbvh_query_vf(uint32_t n_leaves, const float* node_aabb8, const uint32_t* children2,
                           const uint32_t* object_idx, const float* x0, const float* x1,
                           uint32_t n_verts, const float* dhat, const float* thickness,
                           uint32_t* pairs, uint32_t capacity)
{
    if (n_leaves == 0) return 0;
    int nt = NTHREADS;
    pairbuf* bufs = (pairbuf*)calloc((size_t)nt, sizeof(pairbuf));
#pragma omp parallel
    {
        uint32_t tmp[2 * 4096];
        pairbuf* b = &bufs[TID];
#pragma omp for schedule(dynamic, 256)
        for (long long vl = 0; vl < (long long)n_verts; ++vl) {
            uint32_t v = (uint32_t)vl;
            if (dhat[v] < 0.0f) continue; /* affine-body DOF slot: no queries */
            v3_f a = ld3(x0, v), c = ld3(x1, v);
            float r = thickness[v] + dhat[v];
            float q[8] = {fminf_(a.x, c.x) - r, fminf_(a.y, c.y) - r, fminf_(a.z, c.z) - r, 0,
                          fmaxf_(a.x, c.x) + r, fmaxf_(a.y, c.y) + r, fmaxf_(a.z, c.z) + r, 0};
            uint32_t cnt = query_one(node_aabb8, children2, object_idx, q, v, 0xFFFFFFFFu, tmp, 4096);
            if (cnt > 4096) cnt = 4096;
            push_pairs(b, tmp, cnt);
        }
    }
    uint32_t total = gather_pairs(bufs, nt, pairs, capacity);
    free(bufs);
    return total;
}

/* fn_query_from_edges_v2, lbvh.cpp:810-846: swept box of the edge +- (thickness + d_hat) of its
 * first vertex; only eid < adj_eid is kept */
uint32_t orc_lbvh_query_ee(uint32_t n_leaves, const float* node_aabb8, const uint32_t* children2,
                           const uint32_t* object_idx, const float* x0, const float* x1,
                           const uint32_t* edges, uint32_t n_edges, const float* dhat,
                           const float* thickness, uint32_t* pairs, uint32_t capacity)
{
    if (n_leaves == 0) return 0;
    int nt = NTHREADS;
    pairbuf* bufs = (pairbuf*)calloc((size_t)nt, sizeof(pairbuf));
#pragma omp parallel
    {
        uint32_t tmp[2 * 4096];
        pairbuf* b = &bufs[TID];
#pragma omp for schedule(dynamic, 256)
        for (long long el = 0; el < (long long)n_edges; ++el) {
            uint32_t e = (uint32_t)el;
            uint32_t v0 = edges[2 * (size_t)e], v1 = edges[2 * (size_t)e + 1];
            v3_f s0 = ld3(x0, v0), s1 = ld3(x0, v1), e0 = ld3(x1, v0), e1 = ld3(x1, v1);
            float r = thickness[v0] + dhat[v0];
            float q[8] = {fminf_(fminf_(s0.x, s1.x), fminf_(e0.x, e1.x)) - r,
                          fminf_(fminf_(s0.y, s1.y), fminf_(e0.y, e1.y)) - r,
                          fminf_(fminf_(s0.z, s1.z), fminf_(e0.z, e1.z)) - r, 0,
                          fmaxf_(fmaxf_(s0.x, s1.x), fmaxf_(e0.x, e1.x)) + r,
                          fmaxf_(fmaxf_(s0.y, s1.y), fmaxf_(e0.y, e1.y)) + r,
                          fmaxf_(fmaxf_(s0.z, s1.z), fmaxf_(e0.z, e1.z)) + r, 0};
            uint32_t cnt = query_one(node_aabb8, children2, object_idx, q, e, e, tmp, 4096);
            if (cnt > 4096) cnt = 4096;
            push_pairs(b, tmp, cnt);
        }
    }
    uint32_t total = gather_pairs(bufs, nt, pairs, capacity);
    free(bufs);
    return total;
}

/* =========================================================================================
 * ACCD  (Solver/CollisionDetector/accd.hpp:31-205)
 * ========================================================================================= */

/* accd.hpp:31-43 */
static void centerize(v3_f* x)
{
    v3_f mov = mk_f(0.0f, 0.0f, 0.0f);
    for (int k = 0; k < 4; ++k) mov = add_f(mov, scl_f(0.25f, x[k]));
    for (int k = 0; k < 4; ++k) x[k] = sub_f(x[k], mov);
}

/* accd.hpp:129-141 */
static float max_relative_u(const v3_f* u)
{
    float m = 0.0f;
    for (int i = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j) {
            v3_f du = sub_f(u[i], u[j]);
            m = fmaxf_(m, dot_f(du, du));
        }
    return sqrtf(m);
}

/*
 * ccd_helper, accd.hpp:49-101.  fp64_final (the precision form): when the loop stops at a
 * contact bound, the distance at that toi is re-evaluated in FP64; if it does not clear the
 * offset, the previous (smaller) iterate is returned, and the result is rounded one ulp down.
 */
static float ccd_helper(const v3_f* x0, const v3_f* dx, float u_max, int is_ee, float offset,
                        int fp64_final)
{
    float toi = 0.0f, prev = 0.0f;
    const float max_t = 1.25f;
    float eps = 0.01f * (sqrtf(dist2_of_f(is_ee, x0)) - offset);
    float target = eps + offset;
    float eps_sqr = eps * eps;
    float inv_u_max = 1.0f / u_max;
    unsigned iter = 0;
    int contact = 0;
    for (;;) {
        if (iter > 10000u) { toi = 0.001f; break; }
        iter++;
        v3_f xt[4];
        for (int k = 0; k < 4; ++k) xt[k] = add_f(x0[k], scl_f(toi, dx[k]));
        float d2 = dist2_of_f(is_ee, xt);
        float dmt = (d2 - target * target) / (sqrtf(d2) + target);
        if ((max_t - toi) * u_max < dmt - eps) { toi = max_t; break; }
        else if (toi > 0.0f && dmt * dmt < eps_sqr) { contact = 1; break; }
        float toi_next = toi + dmt * inv_u_max;
        if (toi_next != toi) { prev = toi; toi = toi_next; }
        else { contact = 1; break; }
        if (toi > max_t) { toi = max_t; break; }
    }
    if (fp64_final && contact && toi > 0.0f) {
        v3_d xd[4];
        for (int k = 0; k < 4; ++k)
            xd[k] = add_d(mk_d(x0[k].x, x0[k].y, x0[k].z), scl_d((double)toi, mk_d(dx[k].x, dx[k].y, dx[k].z)));
        double d = sqrt(dist2_of_d(is_ee, xd));
        if (!(d > (double)offset)) toi = prev;
        toi = nextafterf(toi, 0.0f);
    }
    return toi;
}

/* accd.hpp:143-171 */
float orc_point_triangle_ccd(const float* p0, const float* p1, const float* t00, const float* t01,
                             const float* t02, const float* t10, const float* t11,
                             const float* t12, float offset, int fp64_final)
{
    v3_f x0[4] = {ldp(p0), ldp(t00), ldp(t01), ldp(t02)};
    v3_f dx[4] = {sub_f(ldp(p1), ldp(p0)), sub_f(ldp(t10), ldp(t00)), sub_f(ldp(t11), ldp(t01)),
                  sub_f(ldp(t12), ldp(t02))};
    centerize(x0);
    centerize(dx);
    float u_max = max_relative_u(dx);
    float toi = 1.25f;
    if (u_max != 0.0f) toi = ccd_helper(x0, dx, u_max, 0, offset, fp64_final);
    return toi;
}

/* accd.hpp:173-202 */
float orc_edge_edge_ccd(const float* ea00, const float* ea01, const float* eb00, const float* eb01,
                        const float* ea10, const float* ea11, const float* eb10, const float* eb11,
                        float offset, int fp64_final)
{
    v3_f x0[4] = {ldp(ea00), ldp(ea01), ldp(eb00), ldp(eb01)};
    v3_f dx[4] = {sub_f(ldp(ea10), ldp(ea00)), sub_f(ldp(ea11), ldp(ea01)), sub_f(ldp(eb10), ldp(eb00)),
                  sub_f(ldp(eb11), ldp(eb01))};
    centerize(x0);
    centerize(dx);
    float u_max = max_relative_u(dx);
    float toi = 1.25f;
    if (u_max != 0.0f) toi = ccd_helper(x0, dx, u_max, 1, offset, fp64_final);
    return toi;
}

/* ---- all-FP64 ACCD: the same algorithm with every quantity in double (the error reference of
 * the precision form; inputs are the FP32 positions promoted exactly) ---- */
static void centerize_d(v3_d* x)
{
    v3_d mov = mk_d(0.0, 0.0, 0.0);
    for (int k = 0; k < 4; ++k) mov = add_d(mov, scl_d(0.25, x[k]));
    for (int k = 0; k < 4; ++k) x[k] = sub_d(x[k], mov);
}

static double ccd_helper_d(const v3_d* x0, const v3_d* dx, double u_max, int is_ee, double offset)
{
    double toi = 0.0;
    const double max_t = 1.25;
    double eps = 0.01 * (sqrt(dist2_of_d(is_ee, x0)) - offset);
    double target = eps + offset, eps_sqr = eps * eps, inv_u_max = 1.0 / u_max;
    for (unsigned iter = 0;; ++iter) {
        if (iter > 10000u) return 0.001;
        v3_d xt[4];
        for (int k = 0; k < 4; ++k) xt[k] = add_d(x0[k], scl_d(toi, dx[k]));
        double d2 = dist2_of_d(is_ee, xt);
        double dmt = (d2 - target * target) / (sqrt(d2) + target);
        if ((max_t - toi) * u_max < dmt - eps) return max_t;
        if (toi > 0.0 && dmt * dmt < eps_sqr) break;
        double nt = toi + dmt * inv_u_max;
        if (nt == toi) break;
        toi = nt;
        if (toi > max_t) return max_t;
    }
    return toi;
}

double orc_ccd_f64(int is_ee, const float* a0, const float* a1, const float* a2, const float* a3,
                   const float* b0, const float* b1, const float* b2, const float* b3, float offset)
{
    const float* A[4] = {a0, a1, a2, a3};
    const float* Bv[4] = {b0, b1, b2, b3};
    v3_d x0[4], dx[4];
    for (int k = 0; k < 4; ++k) {
        x0[k] = mk_d(A[k][0], A[k][1], A[k][2]);
        dx[k] = sub_d(mk_d(Bv[k][0], Bv[k][1], Bv[k][2]), x0[k]);
    }
    centerize_d(x0);
    centerize_d(dx);
    double m = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j) {
            v3_d du = sub_d(dx[i], dx[j]);
            double q = dot_d(du, du);
            if (q > m) m = q;
        }
    double u_max = sqrt(m);
    if (u_max == 0.0) return 1.25;
    return ccd_helper_d(x0, dx, u_max, is_ee, (double)offset);
}

/* per-pair FP64 TOI over a candidate list (VF: vid, fid over faces; EE: edge pairs) */
void orc_ccd_f64_list(int is_ee, const uint32_t* pairs, uint32_t n_pairs, const float* x0, const float* x1,
                      const uint32_t* elems, const uint32_t* body, const float* offset, double* toi)
{
#pragma omp parallel for schedule(dynamic, 1024)
    for (long long pl = 0; pl < (long long)n_pairs; ++pl) {
        uint32_t v[4];
        int skip;
        if (is_ee) {
            uint32_t l = pairs[2 * pl], r = pairs[2 * pl + 1];
            v[0] = elems[2 * (size_t)l]; v[1] = elems[2 * (size_t)l + 1];
            v[2] = elems[2 * (size_t)r]; v[3] = elems[2 * (size_t)r + 1];
            skip = v[0] == v[2] || v[0] == v[3] || v[1] == v[2] || v[1] == v[3] ||
                   (body[v[0]] != 0xFFFFFFFFu && body[v[0]] == body[v[2]]);
        } else {
            uint32_t f = pairs[2 * pl + 1];
            v[0] = pairs[2 * pl];
            v[1] = elems[4 * (size_t)f]; v[2] = elems[4 * (size_t)f + 1]; v[3] = elems[4 * (size_t)f + 2];
            skip = v[0] == v[1] || v[0] == v[2] || v[0] == v[3] ||
                   (body[v[0]] != 0xFFFFFFFFu && body[v[0]] == body[v[1]]);
        }
        if (skip) { toi[pl] = 1.25; continue; }
        float th = offset[v[0]] + offset[is_ee ? v[2] : v[1]];
        toi[pl] = orc_ccd_f64(is_ee, x0 + 4 * (size_t)v[0], x0 + 4 * (size_t)v[1], x0 + 4 * (size_t)v[2],
                              x0 + 4 * (size_t)v[3], x1 + 4 * (size_t)v[0], x1 + 4 * (size_t)v[1],
                              x1 + 4 * (size_t)v[2], x1 + 4 * (size_t)v[3], th);
    }
}

float orc_pt_dist2(const float* p, const float* t0, const float* t1, const float* t2)
{
    return pt_dist2_f(ldp(p), ldp(t0), ldp(t1), ldp(t2));
}
float orc_ee_dist2(const float* a0, const float* a1, const float* b0, const float* b1)
{
    return ee_dist2_f(ldp(a0), ldp(a1), ldp(b0), ldp(b1));
}
void orc_pt_coeff(const float* p, const float* t0, const float* t1, const float* t2, float* c3)
{
    pt_coeff_f(ldp(p), ldp(t0), ldp(t1), ldp(t2), c3);
}
void orc_ee_coeff(const float* a0, const float* a1, const float* b0, const float* b1, float* c4)
{
    ee_coeff_f(ldp(a0), ldp(a1), ldp(b0), ldp(b1), c4);
}

/* ipc::barrier and its derivatives, cipc_kernel.hpp:16-36 */
static inline float barrier_f(float d, float dhat)
{
    float t = d - dhat;
    return -t * t * logf(d / dhat);
}
static inline float barrier_d1(float d, float dhat)
{
    return (dhat - d) * (2.0f * logf(d / dhat) - dhat / d + 1.0f);
}
static inline float barrier_d2(float d, float dhat)
{
    float q = dhat / d;
    return (q + 2.0f) * q - 2.0f * logf(d / dhat) - 3.0f;
}
void orc_barrier(float d, float dhat, float* b, float* db, float* ddb)
{
    *b = barrier_f(d, dhat);
    *db = barrier_d1(d, dhat);
    *ddb = barrier_d2(d, dhat);
}

/* =========================================================================================
 * Narrow phase  (Solver/CollisionDetector/narrow_phase.cpp)
 * ========================================================================================= */

/*
 * fn_narrow_phase_vf_ccd_query, narrow_phase.cpp:293-436.  Incident or same-rigid-body pairs
 * keep toi = 1.25.  Global result (block min -> atomic_min(toi[0], toi / 1.25) on a slot
 * reset to 1.0) is min(1, min_p toi_p / 1.25).
 */
float orc_ccd_vf(const uint32_t* pairs, uint32_t n_pairs, const float* x0, const float* x1,
                 const uint32_t* faces, const uint32_t* body, const float* offset,
                 float* toi_per_pair, int fp64_final)
{
    float gmin = 1.0f;
#pragma omp parallel for schedule(dynamic, 1024) reduction(min : gmin)
    for (long long pl = 0; pl < (long long)n_pairs; ++pl) {
        uint32_t vid = pairs[2 * pl], fid = pairs[2 * pl + 1];
        uint32_t f0 = faces[4 * (size_t)fid], f1 = faces[4 * (size_t)fid + 1], f2 = faces[4 * (size_t)fid + 2];
        float toi = 1.25f;
        int skip = vid == f0 || vid == f1 || vid == f2 ||
                   (body[vid] != 0xFFFFFFFFu && body[vid] == body[f0]);
        if (!skip) {
            float th = offset[vid] + offset[f0];
            toi = orc_point_triangle_ccd(x0 + 4 * (size_t)vid, x1 + 4 * (size_t)vid, x0 + 4 * (size_t)f0,
                                         x0 + 4 * (size_t)f1, x0 + 4 * (size_t)f2, x1 + 4 * (size_t)f0,
                                         x1 + 4 * (size_t)f1, x1 + 4 * (size_t)f2, th, fp64_final);
        }
        if (toi_per_pair) toi_per_pair[pl] = toi;
        float g = toi / 1.25f;
        if (g < gmin) gmin = g;
    }
    return gmin;
}

/* fn_narrow_phase_ee_ccd_query, narrow_phase.cpp:438-593 */
float orc_ccd_ee(const uint32_t* pairs, uint32_t n_pairs, const float* x0, const float* x1,
                 const uint32_t* edges, const uint32_t* body, const float* offset,
                 float* toi_per_pair, int fp64_final)
{
    float gmin = 1.0f;
#pragma omp parallel for schedule(dynamic, 1024) reduction(min : gmin)
    for (long long pl = 0; pl < (long long)n_pairs; ++pl) {
        uint32_t l = pairs[2 * pl], r = pairs[2 * pl + 1];
        uint32_t a0 = edges[2 * (size_t)l], a1 = edges[2 * (size_t)l + 1];
        uint32_t b0 = edges[2 * (size_t)r], b1 = edges[2 * (size_t)r + 1];
        float toi = 1.25f;
        int skip = a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1 ||
                   (body[a0] != 0xFFFFFFFFu && body[a0] == body[b0]);
        if (!skip) {
            float th = offset[a0] + offset[b0];
            toi = orc_edge_edge_ccd(x0 + 4 * (size_t)a0, x0 + 4 * (size_t)a1, x0 + 4 * (size_t)b0,
                                    x0 + 4 * (size_t)b1, x1 + 4 * (size_t)a0, x1 + 4 * (size_t)a1,
                                    x1 + 4 * (size_t)b0, x1 + 4 * (size_t)b1, th, fp64_final);
        }
        if (toi_per_pair) toi_per_pair[pl] = toi;
        float g = toi / 1.25f;
        if (g < gmin) gmin = g;
    }
    return gmin;
}

/* CollisionPairTemplate::make_vf_pair / make_ee_pair, collision_data.h:169-193 (type bit 31 on
 * idx[2] for VF, idx[3] for EE) */
static void make_pair(orc_pair* p, uint32_t i0, uint32_t i1, uint32_t i2, uint32_t i3, int is_ee,
                      v3_f n, float k1, float k2, float stiff, float b0, float b1)
{
    p->idx[0] = i0; p->idx[1] = i1; p->idx[2] = i2; p->idx[3] = i3;
    if (is_ee) p->idx[3] |= 0x80000000u; else p->idx[2] |= 0x80000000u;
    p->vec1[0] = n.x; p->vec1[1] = n.y; p->vec1[2] = n.z; p->vec1[3] = stiff;
    p->vec2[0] = k1; p->vec2[1] = k2; p->vec2[2] = b0; p->vec2[3] = b1;
}

/* fn_narrow_phase_vf_dcd_query (barrier energy), narrow_phase.cpp:771-933 */
uint32_t orc_dcd_vf(const uint32_t* pairs, uint32_t n_pairs, const float* x, const uint32_t* faces,
                    const uint32_t* body, const float* vert_area, const float* face_area,
                    const float* dhat_v, const float* offset, float kappa, orc_pair* out,
                    uint32_t capacity)
{
    uint32_t count = 0;
    for (uint32_t pl = 0; pl < n_pairs; ++pl) {
        uint32_t vid = pairs[2 * (size_t)pl], fid = pairs[2 * (size_t)pl + 1];
        uint32_t f0 = faces[4 * (size_t)fid], f1 = faces[4 * (size_t)fid + 1], f2 = faces[4 * (size_t)fid + 2];
        if (vid == f0 || vid == f1 || vid == f2 || (body[vid] != 0xFFFFFFFFu && body[vid] == body[f0]))
            continue;
        v3_f p = ld3(x, vid), t0 = ld3(x, f0), t1 = ld3(x, f1), t2 = ld3(x, f2);
        float c[3];
        pt_coeff_f(p, t0, t1, t2, c);
        v3_f xv = add_f(add_f(scl_f(c[0], sub_f(p, t0)), scl_f(c[1], sub_f(p, t1))), scl_f(c[2], sub_f(p, t2)));
        float d2 = dot_f(xv, xv);
        float dh = (dhat_v[vid] + dhat_v[f0]) * 0.5f;
        float th = offset[vid] + offset[f0];
        float lim = th + dh;
        if (d2 < lim * lim) {
            float d = sqrtf(d2);
            v3_f n = mk_f(xv.x / d, xv.y / d, xv.z / d);
            float area = 0.5f * (vert_area[vid] + face_area[fid]);
            float k1 = -area * kappa * barrier_d1(d - th, dh);
            float k2 = area * kappa * barrier_d2(d - th, dh);
            if (count < capacity) make_pair(&out[count], vid, f0, f1, f2, 0, n, k1, k2, area * kappa, c[0], c[1]);
            count++;
        }
    }
    return count;
}

/* fn_narrow_phase_ee_dcd_query (barrier energy), narrow_phase.cpp:935-1098 */
uint32_t orc_dcd_ee(const uint32_t* pairs, uint32_t n_pairs, const float* x, const uint32_t* edges,
                    const uint32_t* body, const float* edge_area, const float* dhat_v,
                    const float* offset, float kappa, orc_pair* out, uint32_t capacity)
{
    uint32_t count = 0;
    for (uint32_t pl = 0; pl < n_pairs; ++pl) {
        uint32_t l = pairs[2 * (size_t)pl], r = pairs[2 * (size_t)pl + 1];
        uint32_t a0 = edges[2 * (size_t)l], a1 = edges[2 * (size_t)l + 1];
        uint32_t b0 = edges[2 * (size_t)r], b1 = edges[2 * (size_t)r + 1];
        if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1 || (body[a0] != 0xFFFFFFFFu && body[a0] == body[b0]))
            continue;
        v3_f ea0 = ld3(x, a0), ea1 = ld3(x, a1), eb0 = ld3(x, b0), eb1 = ld3(x, b1);
        float c[4];
        ee_coeff_f(ea0, ea1, eb0, eb1, c);
        v3_f x0 = add_f(scl_f(c[0], ea0), scl_f(c[1], ea1));
        v3_f x1 = add_f(scl_f(c[2], eb0), scl_f(c[3], eb1));
        v3_f xv = sub_f(x0, x1);
        float d2 = dot_f(xv, xv);
        float dh = (dhat_v[a0] + dhat_v[b0]) * 0.5f;
        float th = offset[a0] + offset[b0];
        float lim = th + dh;
        if (d2 < lim * lim) {
            float d = sqrtf(d2);
            v3_f n = mk_f(xv.x / d, xv.y / d, xv.z / d);
            float area = 0.5f * (edge_area[l] + edge_area[r]);
            float k1 = -area * kappa * barrier_d1(d - th, dh);
            float k2 = area * kappa * barrier_d2(d - th, dh);
            if (count < capacity) make_pair(&out[count], a0, a1, b0, b1, 1, n, k1, k2, area * kappa, c[0], c[2]);
            count++;
        }
    }
    return count;
}

/* CollisionPairTemplate::get_weight, collision_data.h:308-324 */
static inline int pair_weights(const orc_pair* p, uint32_t* v, float* w)
{
    for (int k = 0; k < 4; ++k) v[k] = p->idx[k] & 0x7FFFFFFFu;
    int is_vf = (p->idx[2] >> 31) & 1u, is_ee = (p->idx[3] >> 31) & 1u;
    float b0 = p->vec2[2], b1 = p->vec2[3];
    if (is_vf) { w[0] = 1.0f; w[1] = -b0; w[2] = -b1; w[3] = b0 + b1 - 1.0f; return 1; }
    if (is_ee) { w[0] = b0; w[1] = 1.0f - b0; w[2] = -b1; w[3] = b1 - 1.0f; return 2; }
    w[0] = w[1] = w[2] = w[3] = 0.0f;
    return 0;
}

/* fn_perPair_assemble_gradient_hessian, narrow_phase.cpp:2550-2676 (soft bodies):
 * b[v_i] += (k1 w_i) n ; D[v_i] += ((k2 w_i) w_i) n n^T.  diag12 = 3 float4 columns. */
void orc_contact_grad_diag(const orc_pair* pairs, uint32_t n, float* b4, float* diag12)
{
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t v[4];
        float w[4];
        if (!pair_weights(&pairs[k], v, w)) continue;
        float nx = pairs[k].vec1[0], ny = pairs[k].vec1[1], nz = pairs[k].vec1[2];
        float k1 = pairs[k].vec2[0], k2 = pairs[k].vec2[1];
        float nn[3] = {nx, ny, nz};
        for (int i = 0; i < 4; ++i) {
            float g = k1 * w[i];
            b4[4 * (size_t)v[i] + 0] += g * nx;
            b4[4 * (size_t)v[i] + 1] += g * ny;
            b4[4 * (size_t)v[i] + 2] += g * nz;
            float h = k2 * w[i] * w[i];
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) diag12[12 * (size_t)v[i] + 4 * c + r] += h * (nn[r] * nn[c]);
        }
    }
}

typedef struct { uint64_t key; uint32_t pair; uint8_t i, j; } trip;
static int cmp_trip(const void* a, const void* b)
{
    const trip* x = (const trip*)a;
    const trip* y = (const trip*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    if (x->pair != y->pair) return x->pair < y->pair ? -1 : 1;
    if (x->i != y->i) return x->i < y->i ? -1 : 1;
    return x->j < y->j ? -1 : (x->j > y->j ? 1 : 0);
}

/*
 * Off-diagonal contact blocks (fn_fill_in_pairs_in_vert_adjacent + the triplet sort +
 * fn_assemble_triplet_sorted, narrow_phase.cpp:1317-1386, 1434-1880): every ordered pair
 * (v_i, v_j), i != j, of a soft-soft pair adds (w_i w_j)(k2 n n^T); equal (row, col) keys are
 * summed.  The result is BSR: row_ptr[n_rows + 1], col, 9 floats per block (column-major),
 * blocks in (row, col) order.  Returns the number of blocks (may exceed cap: then nothing is
 * written beyond cap and the caller retries with the returned size).
 */
uint32_t orc_contact_offdiag_bsr(const orc_pair* pairs, uint32_t n, uint32_t n_rows,
                                 uint32_t* row_ptr, uint32_t* col, float* val9, uint32_t cap)
{
    trip* t = (trip*)malloc(sizeof(trip) * 12 * (size_t)(n ? n : 1));
    size_t nt = 0;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t v[4];
        float w[4];
        if (!pair_weights(&pairs[k], v, w)) continue;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                if (i != j) {
                    t[nt].key = ((uint64_t)v[i] << 32) | v[j];
                    t[nt].pair = k;
                    t[nt].i = (uint8_t)i;
                    t[nt].j = (uint8_t)j;
                    nt++;
                }
    }
    qsort(t, nt, sizeof(trip), cmp_trip);
    uint32_t nb = 0;
    for (uint32_t r = 0; r <= n_rows; ++r) row_ptr[r] = 0;
    for (size_t s = 0; s < nt; ++s) {
        if (s == 0 || t[s].key != t[s - 1].key) {
            uint32_t row = (uint32_t)(t[s].key >> 32);
            if (nb < cap) {
                col[nb] = (uint32_t)(t[s].key & 0xFFFFFFFFu);
                for (int q = 0; q < 9; ++q) val9[9 * (size_t)nb + q] = 0.0f;
            }
            if (row < n_rows) row_ptr[row + 1]++;
            nb++;
        }
        if (nb - 1 < cap) {
            const orc_pair* p = &pairs[t[s].pair];
            uint32_t v[4];
            float w[4];
            pair_weights(p, v, w);
            float k2 = p->vec2[1];
            float nn[3] = {p->vec1[0], p->vec1[1], p->vec1[2]};
            float sw = w[t[s].i] * w[t[s].j];
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) val9[9 * (size_t)(nb - 1) + 3 * c + r] += sw * (k2 * (nn[r] * nn[c]));
        }
    }
    for (uint32_t r = 0; r < n_rows; ++r) row_ptr[r + 1] += row_ptr[r];
    free(t);
    return nb;
}

/*
 * Affine bodies: the generalised DOFs of a pair (get_active_indices, collision_data.h:198-268, and
 * add_to_rigid_body, narrow_phase.cpp:2612-2629).  Each side (VF: vertex 0 | face 1..3; EE: edge 0,1 | edge
 * 2,3) is soft -- its vertices and weights -- or rigid -- its body's four DOF slots body_dof[b] + j with
 * weights sum_i w_i (1, x_bar_i), the body being that of vertex 0 (left) or vertex 2 (right).
 */
static int pair_dofs_abd(const orc_pair* p, const uint32_t* body, const float* model_x4, const uint32_t* body_dof,
                         uint32_t dof[8], float gw[8])
{
    uint32_t v[4];
    float w[4];
    if (!pair_weights(p, v, w)) return 0;
    const int split = (p->idx[2] >> 31) ? 1 : 2;
    int n = 0;
    for (int side = 0; side < 2; ++side) {
        const int s0 = side ? split : 0, s1 = side ? 4 : split;
        const uint32_t b = body[v[side ? 2 : 0]];
        if (b == 0xFFFFFFFFu) {
            for (int i = s0; i < s1; ++i) {
                dof[n] = v[i];
                gw[n] = w[i];
                ++n;
            }
        } else {
            float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
            for (int i = s0; i < s1; ++i) {
                const float* m = model_x4 + 4 * (size_t)v[i];
                a0 += w[i];
                a1 += w[i] * m[0];
                a2 += w[i] * m[1];
                a3 += w[i] * m[2];
            }
            const float aw[4] = {a0, a1, a2, a3};
            for (int j = 0; j < 4; ++j) {
                dof[n] = body_dof[b] + (uint32_t)j;
                gw[n] = aw[j];
                ++n;
            }
        }
    }
    return n;
}

void orc_contact_grad_diag_abd(const orc_pair* pairs, uint32_t n, const uint32_t* body, const float* model_x4,
                               const uint32_t* body_dof, float* b4, float* diag12)
{
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t dof[8];
        float gw[8];
        const int nd = pair_dofs_abd(&pairs[k], body, model_x4, body_dof, dof, gw);
        float nx = pairs[k].vec1[0], ny = pairs[k].vec1[1], nz = pairs[k].vec1[2];
        float k1 = pairs[k].vec2[0], k2 = pairs[k].vec2[1];
        float nn[3] = {nx, ny, nz};
        for (int i = 0; i < nd; ++i) {
            float g = k1 * gw[i];
            b4[4 * (size_t)dof[i] + 0] += g * nx;
            b4[4 * (size_t)dof[i] + 1] += g * ny;
            b4[4 * (size_t)dof[i] + 2] += g * nz;
            float h = k2 * gw[i] * gw[i];
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) diag12[12 * (size_t)dof[i] + 4 * c + r] += h * (nn[r] * nn[c]);
        }
    }
}

/* orc_contact_offdiag_bsr over the generalised DOFs (every ordered pair of a pair's DOFs) */
uint32_t orc_contact_offdiag_bsr_abd(const orc_pair* pairs, uint32_t n, uint32_t n_rows, const uint32_t* body,
                                     const float* model_x4, const uint32_t* body_dof, uint32_t* row_ptr, uint32_t* col,
                                     float* val9, uint32_t cap)
{
    trip* t = (trip*)malloc(sizeof(trip) * 56 * (size_t)(n ? n : 1));
    size_t nt = 0;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t dof[8];
        float gw[8];
        const int nd = pair_dofs_abd(&pairs[k], body, model_x4, body_dof, dof, gw);
        for (int i = 0; i < nd; ++i)
            for (int j = 0; j < nd; ++j)
                if (i != j) {
                    t[nt].key = ((uint64_t)dof[i] << 32) | dof[j];
                    t[nt].pair = k;
                    t[nt].i = (uint8_t)i;
                    t[nt].j = (uint8_t)j;
                    nt++;
                }
    }
    qsort(t, nt, sizeof(trip), cmp_trip);
    uint32_t nb = 0;
    for (uint32_t r = 0; r <= n_rows; ++r) row_ptr[r] = 0;
    for (size_t s = 0; s < nt; ++s) {
        if (s == 0 || t[s].key != t[s - 1].key) {
            uint32_t row = (uint32_t)(t[s].key >> 32);
            if (nb < cap) {
                col[nb] = (uint32_t)(t[s].key & 0xFFFFFFFFu);
                for (int q = 0; q < 9; ++q) val9[9 * (size_t)nb + q] = 0.0f;
            }
            if (row < n_rows) row_ptr[row + 1]++;
            nb++;
        }
        if (nb - 1 < cap) {
            const orc_pair* p = &pairs[t[s].pair];
            uint32_t dof[8];
            float gw[8];
            pair_dofs_abd(p, body, model_x4, body_dof, dof, gw);
            float k2 = p->vec2[1];
            float nn[3] = {p->vec1[0], p->vec1[1], p->vec1[2]};
            float sw = gw[t[s].i] * gw[t[s].j];
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) val9[9 * (size_t)(nb - 1) + 3 * c + r] += sw * (k2 * (nn[r] * nn[c]));
        }
    }
    for (uint32_t r = 0; r < n_rows; ++r) row_ptr[r + 1] += row_ptr[r];
    free(t);
    return nb;
}

/* fn_compute_repulsion_energy (barrier), narrow_phase.cpp:2968-3044 */
double orc_contact_energy(const orc_pair* pairs, uint32_t n, const float* x, const float* dhat_v,
                          const float* offset, int fp64_sum)
{
    double sd = 0.0;
    float sf = 0.0f;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t v[4];
        float w[4];
        if (!pair_weights(&pairs[k], v, w)) continue;
        v3_f diff = add_f(add_f(add_f(scl_f(w[0], ld3(x, v[0])), scl_f(w[1], ld3(x, v[1]))),
                                scl_f(w[2], ld3(x, v[2]))),
                          scl_f(w[3], ld3(x, v[3])));
        float d = sqrtf(dot_f(diff, diff));
        float dh = 0.5f * (dhat_v[v[0]] + dhat_v[v[2]]);
        float th = offset[v[0]] + offset[v[2]];
        float e = 0.0f;
        if (d < th + dh) e = pairs[k].vec1[3] * barrier_f(d - th, dh);
        sd += (double)e;
        sf += e;
    }
    return fp64_sum ? sd : (double)sf;
}

/* =========================================================================================
 * SpMV + Jacobi PCG  (newton_solver.cpp:259-472, 3397-3427; precond_cg.cpp:33-331, 626-771)
 * ========================================================================================= */

static inline void mv9(const float* m, const float* x, float* y)
{
    for (int r = 0; r < 3; ++r) y[r] = fmaf(m[6 + r], x[2], fmaf(m[3 + r], x[1], m[r] * x[0]));
}
static inline void mv12(const float* m, const float* x, float* y)
{
    for (int r = 0; r < 3; ++r) y[r] = fmaf(m[8 + r], x[2], fmaf(m[4 + r], x[1], m[r] * x[0]));
}

/* device_SpMV: y = D x + A_offdiag x + B_offdiag x (B may be absent) */
void orc_bsr_spmv(uint32_t n, const float* diag12, const uint32_t* rp_a, const uint32_t* col_a,
                  const float* val_a, const uint32_t* rp_b, const uint32_t* col_b,
                  const float* val_b, const float* x4, float* y4)
{
#pragma omp parallel for schedule(static)
    for (long long il = 0; il < (long long)n; ++il) {
        uint32_t i = (uint32_t)il;
        float acc[3], t[3];
        mv12(diag12 + 12 * (size_t)i, x4 + 4 * (size_t)i, acc);
        if (rp_a)
            for (uint32_t k = rp_a[i]; k < rp_a[i + 1]; ++k) {
                mv9(val_a + 9 * (size_t)k, x4 + 4 * (size_t)col_a[k], t);
                acc[0] += t[0]; acc[1] += t[1]; acc[2] += t[2];
            }
        if (rp_b)
            for (uint32_t k = rp_b[i]; k < rp_b[i + 1]; ++k) {
                mv9(val_b + 9 * (size_t)k, x4 + 4 * (size_t)col_b[k], t);
                acc[0] += t[0]; acc[1] += t[1]; acc[2] += t[2];
            }
        y4[4 * (size_t)i + 0] = acc[0];
        y4[4 * (size_t)i + 1] = acc[1];
        y4[4 * (size_t)i + 2] = acc[2];
        y4[4 * (size_t)i + 3] = 0.0f;
    }
}

/* inverse() of a 3x3 (adjugate / determinant), used by fn_pcg_make_preconditioner */
static void inv3(const float* m, float* o)
{
    /* m column-major with float4 columns: m[4c + r] */
    float a = m[0], b = m[4], c = m[8];
    float d = m[1], e = m[5], f = m[9];
    float g = m[2], h = m[6], k = m[10];
    float A = e * k - f * h, B = f * g - d * k, C = d * h - e * g;
    float det = a * A + b * B + c * C;
    float id = 1.0f / det;
    /* inverse rows: [A, c h - b k, b f - c e ; B, a k - c g, c d - a f ; C, b g - a h, a e - b d] / det */
    float r00 = A * id, r01 = (c * h - b * k) * id, r02 = (b * f - c * e) * id;
    float r10 = B * id, r11 = (a * k - c * g) * id, r12 = (c * d - a * f) * id;
    float r20 = C * id, r21 = (b * g - a * h) * id, r22 = (a * e - b * d) * id;
    o[0] = r00; o[1] = r10; o[2] = r20; o[3] = 0.0f;
    o[4] = r01; o[5] = r11; o[6] = r21; o[7] = 0.0f;
    o[8] = r02; o[9] = r12; o[10] = r22; o[11] = 0.0f;
}

static inline float safe_div(float a, float b) { return b < 1e-10f ? 0.0f : a / b; }

/*
 * ConjugateGradientSolver::device_solve (precond_cg.cpp:626-771) with x0 = 0.  The stop test
 * runs every check_every iterations before p is updated: rz < abs_rz_tol (the reference's
 * 1e-10) or ||r|| <= rel_tol * ||r0|| (rel_tol <= 0 disables it).  fp64_dots selects FP64
 * accumulation of the dot products (precision form); otherwise FP32 in index order.
 */
int orc_pcg(uint32_t n, const float* diag12, const uint32_t* rp_a, const uint32_t* col_a,
            const float* val_a, const uint32_t* rp_b, const uint32_t* col_b, const float* val_b,
            const float* b4, float* x4, int max_iter, float rel_tol, float abs_rz_tol,
            int check_every, int fp64_dots, orc_pcg_stats* stats)
{
    size_t n4 = 4 * (size_t)n;
    float* r = (float*)calloc(n4, sizeof(float));
    float* z = (float*)calloc(n4, sizeof(float));
    float* p = (float*)calloc(n4, sizeof(float));
    float* q = (float*)calloc(n4, sizeof(float));
    float* minv = (float*)calloc(12 * (size_t)n, sizeof(float));
    for (size_t k = 0; k < n4; ++k) { r[k] = b4[k]; x4[k] = 0.0f; }
    for (uint32_t i = 0; i < n; ++i) inv3(diag12 + 12 * (size_t)i, minv + 12 * (size_t)i);
    if (check_every <= 0) check_every = 1;
    float rz_old = 0.0f, norm_r0 = 0.0f, norm_r = 0.0f;
    int iter, status = 0;
    for (iter = 0; iter < max_iter; ++iter) {
        double rr_d = 0.0, rz_d = 0.0;
        float rr_f = 0.0f, rz_f = 0.0f;
        for (uint32_t i = 0; i < n; ++i) {
            float zi[3];
            mv12(minv + 12 * (size_t)i, r + 4 * (size_t)i, zi);
            z[4 * i] = zi[0]; z[4 * i + 1] = zi[1]; z[4 * i + 2] = zi[2];
            float rv[3] = {r[4 * i], r[4 * i + 1], r[4 * i + 2]};
            float drr = fmaf(rv[2], rv[2], fmaf(rv[1], rv[1], rv[0] * rv[0]));
            float drz = fmaf(rv[2], zi[2], fmaf(rv[1], zi[1], rv[0] * zi[0]));
            rr_d += drr; rz_d += drz; rr_f += drr; rz_f += drz;
        }
        float rr = fp64_dots ? (float)rr_d : rr_f;
        float rz = fp64_dots ? (float)rz_d : rz_f;
        float beta = safe_div(rz, rz_old);
        rz_old = rz;
        norm_r = sqrtf(rr);
        if (iter == 0) norm_r0 = norm_r;
        if (iter % check_every == 0) {
            if (isnan(rz) || isinf(rz)) { status = 1; break; }
            if (rz < abs_rz_tol) break;
            if (rel_tol > 0.0f && norm_r <= rel_tol * norm_r0) break;
        }
        for (size_t k = 0; k < n4; ++k) p[k] = z[k] + beta * p[k];
        orc_bsr_spmv(n, diag12, rp_a, col_a, val_a, rp_b, col_b, val_b, p, q);
        double pq_d = 0.0;
        float pq_f = 0.0f;
        for (uint32_t i = 0; i < n; ++i) {
            float d = fmaf(p[4 * i + 2], q[4 * i + 2], fmaf(p[4 * i + 1], q[4 * i + 1], p[4 * i] * q[4 * i]));
            pq_d += d; pq_f += d;
        }
        float pq = fp64_dots ? (float)pq_d : pq_f;
        float alpha = safe_div(rz, pq);
        for (size_t k = 0; k < n4; ++k) {
            x4[k] = x4[k] + alpha * p[k];
            r[k] = r[k] - alpha * q[k];
        }
    }
    if (stats) {
        stats->iterations = iter;
        stats->rel_residual = norm_r0 > 0.0f ? norm_r / norm_r0 : 0.0f;
        stats->dot_rz = rz_old;
        stats->status = status;
    }
    free(r); free(z); free(p); free(q); free(minv);
    return status;
}

/* =========================================================================================
 * Material producers of the Newton loop (inertia + Dirichlet pinning, springs, quadratic
 * bending relative to rest): newton_solver.cpp:819-851, 1003-1045; init_sim_data.cpp:455-480.
 * The off-diagonal pattern is fixed per mesh; spring_slots / bend_slots give each
 * contribution's block.  b = -gradient, diag = 3 float4 columns, val9 column-major.
 * ========================================================================================= */
void orc_material_fill(uint32_t V, uint32_t E, uint32_t B, const float* x4, const float* rest4,
                       const float* xt4, const float* mass, const uint8_t* pinned, float dt,
                       float dirichlet, const uint32_t* edges, const float* rest_len, float spring_k_scalar,
                       const float* spring_kper,
                       const uint32_t* stencil, const float* Q16, float bending_k,
                       const uint32_t* spring_slots, const uint32_t* bend_slots, uint32_t nnz,
                       float* b4, float* diag12, float* val9)
{
    const float h2inv = 1.0f / (dt * dt);
    memset(val9, 0, sizeof(float) * 9 * (size_t)nnz);
#pragma omp parallel for schedule(static)
    for (long long il = 0; il < (long long)V; ++il) {
        size_t i = (size_t)il;
        float m = mass[i], s = -m * h2inv, hd = m * h2inv;
        float g[3];
        for (int k = 0; k < 3; ++k) g[k] = s * (x4[4 * i + k] - xt4[4 * i + k]);
        if (pinned && pinned[i]) {
            for (int k = 0; k < 3; ++k) g[k] = g[k] + dirichlet * g[k];
            hd = hd + dirichlet * hd;
        }
        for (int k = 0; k < 3; ++k) b4[4 * i + k] = g[k];
        b4[4 * i + 3] = 0.0f;
        for (int k = 0; k < 12; ++k) diag12[12 * i + k] = 0.0f;
        diag12[12 * i + 0] = hd;
        diag12[12 * i + 5] = hd;
        diag12[12 * i + 10] = hd;
    }
    for (uint32_t e = 0; e < E; ++e) {
        const float spring_k = spring_kper ? spring_kper[e] : spring_k_scalar;
        uint32_t a = edges[2 * e], c = edges[2 * e + 1];
        float d[3] = {x4[4 * a] - x4[4 * c], x4[4 * a + 1] - x4[4 * c + 1], x4[4 * a + 2] - x4[4 * c + 2]};
        float l = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (l < 1.19209290E-7f) l = 1.19209290E-7f;
        float L = rest_len[e], il = 1.0f / l, il2 = il * il;
        float C = l - L;
        for (int k = 0; k < 3; ++k) {
            float gk = spring_k * d[k] * il * C;
            b4[4 * a + k] -= gk;
            b4[4 * c + k] += gk;
        }
        float aa = spring_k * il2, cc = spring_k * (1.0f - L * il > 0.0f ? 1.0f - L * il : 0.0f);
        float* O0 = val9 + 9 * (size_t)spring_slots[2 * e];
        float* O1 = val9 + 9 * (size_t)spring_slots[2 * e + 1];
        for (int col = 0; col < 3; ++col)
            for (int r = 0; r < 3; ++r) {
                float h = aa * d[r] * d[col] + cc * ((r == col ? 1.0f : 0.0f) - il2 * d[r] * d[col]);
                diag12[12 * (size_t)a + 4 * col + r] += h;
                diag12[12 * (size_t)c + 4 * col + r] += h;
                O0[3 * col + r] -= h;
                O1[3 * col + r] -= h;
            }
    }
    for (uint32_t s = 0; s < B; ++s) {
        const uint32_t* v = stencil + 4 * (size_t)s;
        const float* q = Q16 + 16 * (size_t)s;
        float u[4][3];
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 3; ++k) u[j][k] = x4[4 * (size_t)v[j] + k] - rest4[4 * (size_t)v[j] + k];
        int t = 0;
        for (int i = 0; i < 4; ++i) {
            float g[3] = {0.0f, 0.0f, 0.0f};
            for (int j = 0; j < 4; ++j) {
                float qij = bending_k * q[4 * i + j];
                for (int k = 0; k < 3; ++k) g[k] += qij * u[j][k];
                if (i == j) {
                    diag12[12 * (size_t)v[i] + 0] += qij;
                    diag12[12 * (size_t)v[i] + 5] += qij;
                    diag12[12 * (size_t)v[i] + 10] += qij;
                } else {
                    float* O = val9 + 9 * (size_t)bend_slots[12 * (size_t)s + t];
                    O[0] += qij;
                    O[4] += qij;
                    O[8] += qij;
                    ++t;
                }
            }
            for (int k = 0; k < 3; ++k) b4[4 * (size_t)v[i] + k] -= g[k];
        }
    }
}

/* Smallest unsigned VF / EE distance over candidate pairs (incident pairs skipped): the
 * post-step penetration check (NewtonSolver::device_post_dist_check, newton_solver.cpp:3364-3375). */
float orc_min_distance(const uint32_t* vf, uint32_t n_vf, const uint32_t* ee, uint32_t n_ee, const float* x,
                       const uint32_t* faces, const uint32_t* edges)
{
    float best = 3.402823466e+38F;
#pragma omp parallel for reduction(min : best) schedule(static)
    for (long long k = 0; k < (long long)n_vf; ++k) {
        uint32_t v = vf[2 * k], f = vf[2 * k + 1];
        uint32_t a = faces[4 * (size_t)f], b = faces[4 * (size_t)f + 1], c = faces[4 * (size_t)f + 2];
        if (v == a || v == b || v == c) continue;
        float d = sqrtf(pt_dist2_f(ld3(x, v), ld3(x, a), ld3(x, b), ld3(x, c)));
        if (d < best) best = d;
    }
#pragma omp parallel for reduction(min : best) schedule(static)
    for (long long k = 0; k < (long long)n_ee; ++k) {
        uint32_t l = ee[2 * k], r = ee[2 * k + 1];
        uint32_t a0 = edges[2 * (size_t)l], a1 = edges[2 * (size_t)l + 1];
        uint32_t b0 = edges[2 * (size_t)r], b1 = edges[2 * (size_t)r + 1];
        if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) continue;
        float d = sqrtf(ee_dist2_f(ld3(x, a0), ld3(x, a1), ld3(x, b0), ld3(x, b1)));
        if (d < best) best = d;
    }
    return best;
}
