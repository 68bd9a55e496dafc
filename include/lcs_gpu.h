/*
 * lcs_gpu.h -- C ABI of the B200 (sm_100a) contact-and-solve path of LuisaComputeSimulator.
 *
 * The entry points replace the LuisaCompute shaders behind the reference's LBVH,
 * NarrowPhasesDetector and ConjugateGradientSolver classes (citations per function, paths
 * relative to the reference project).  All pointers are DEVICE pointers unless a parameter
 * says "host"; every call is stream-ordered on the caller's cudaStream_t (NULL = legacy
 * default stream) and returns an lcs_status.  Handles are not thread-safe.
 *
 * Data layouts (identical to LuisaCompute's buffers, so an LC-hosted caller can pass
 * Buffer<T>::native_handle() pointers):
 *   positions   float4 per vertex (x, y, z, pad)                       = Buffer<float3>
 *   faces       uint4  per face   (v0, v1, v2, pad)                     = Buffer<uint3>
 *   edges       uint2  per edge                                         = Buffer<uint2>
 *   diag blocks 3 float4 columns per vertex (48 B)                      = Buffer<float3x3>
 *   BSR blocks  9 floats per block, column-major                        (MatrixTriplet3x3 order)
 *   pairs       lcs_pair, 48 B                                          = CollisionPairTemplate
 *   per-vertex scalars (d_hat, offset, areas) float; body ids uint32 (0xFFFFFFFF = soft)
 */
#ifndef LCS_GPU_H
#define LCS_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LCS_API __attribute__((visibility("default")))
#else
#define LCS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* lcs_stream; /* = cudaStream_t */

typedef enum lcs_status {
    LCS_OK = 0,
    LCS_ERR_INVALID = 1,        /* bad argument (null handle, size mismatch, ...) */
    LCS_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    LCS_ERR_CAPACITY = 3,       /* an output did not fit; the required size was reported */
    LCS_ERR_UNHEALTHY_BVH = 4,  /* parent/child links inconsistent (fn_check_construction) */
    LCS_ERR_NAN = 5,            /* NaN / Inf met (PCG rz, barrier stiffness) */
    LCS_ERR_CCD_NOCONVERGE = 6, /* an ACCD pair hit the 10000-iteration cap (toi 0.001) */
    LCS_ERR_TIMEOUT = 7,        /* a bounded device-side wait gave up */
    LCS_ERR_NO_DEVICE = 8,      /* no CUDA device / not an sm_100 device */
    LCS_ERR_LINESEARCH = 9      /* the energy line search found no decrease above step length 1e-4 */
} lcs_status;

enum { LCS_TREE_VERT = 0, LCS_TREE_EDGE = 1, LCS_TREE_FACE = 2 };

/* flags for the CCD entry points */
enum {
    LCS_CCD_FP64_FINAL = 1, /* FP32 iteration, final iterate re-checked in FP64 (backs off if it fails) */
    LCS_CCD_FP64 = 2        /* the whole iteration in FP64; per-pair TOI rounded toward zero to float */
};

/* CollisionPairTemplate (Solver/SimulationCore/collision_data.h:48-126): indices with the
 * pair type in bit 31 (VF: idx[2], EE: idx[3]); vec1 = (normal, kappa * area);
 * vec2 = (k1, k2, bary0, bary1). */
typedef struct lcs_pair {
    uint32_t idx[4];
    float vec1[4];
    float vec2[4];
} lcs_pair;

/* 3x3-block CSR matrix (device arrays). */
typedef struct lcs_bsr {
    uint32_t n_rows;
    const uint32_t* row_ptr; /* n_rows + 1 */
    const uint32_t* col;     /* nnzb */
    const float* val;        /* 9 * nnzb, column-major blocks */
} lcs_bsr;

/* ------------------------------------------------------------------------------------------
 * Library / device
 * ------------------------------------------------------------------------------------------ */
/* Version string of the library ("lcs_b200 <ver> sm_100a"). Host pointer, static storage. */
LCS_API const char* lcs_version(void);
/* Checks that device `device` is usable (sm_100 family). */
LCS_API int lcs_device_check(int device);
/* Text of the last error recorded on this thread (host pointer, static storage). */
LCS_API const char* lcs_last_error(void);
/* Number of kernels this library has launched in this process (all threads). */
LCS_API uint64_t lcs_launch_count(void);

/* ------------------------------------------------------------------------------------------
 * LBVH  (replaces class LBVH, Solver/CollisionDetector/lbvh.h:166-229)
 * ------------------------------------------------------------------------------------------ */
typedef struct lcs_bvh lcs_bvh;

/* LbvhData::allocate (lbvh.h:95-139): a tree over n_leaves vertices, edges or faces. */
LCS_API int lcs_bvh_create(int kind, uint32_t n_leaves, lcs_bvh** out);
LCS_API int lcs_bvh_destroy(lcs_bvh* h);

/* LBVH::reduce_{vert,edge,face}_tree_aabb (lbvh.cpp:939-973): leaf centres and the global
 * AABB used to normalise Morton codes.  The second pass of the reference covers the first
 * ceil(n_verts / 256) block partials for every tree kind; that is reproduced.
 * elems: NULL (vert tree), uint2 edges (edge tree) or uint4 faces (face tree). */
LCS_API int lcs_bvh_reduce_aabb(lcs_bvh* h, const float* x, const uint32_t* elems, uint32_t n_verts,
                        lcs_stream stream);

/* LBVH::construct_tree (lbvh.cpp:974-998): Morton codes, a device radix sort (the reference
 * sorts on the host), Karras inner nodes, health check.  The health flag stays on the
 * device; read it with lcs_bvh_health. */
LCS_API int lcs_bvh_construct(lcs_bvh* h, lcs_stream stream);

/* LBVH::update_{vert,edge,face}_tree_leave_aabb (lbvh.cpp:1001-1031): swept leaf boxes
 * [x0, x1] +- thickness of the element's first vertex.  This, the two refit calls below, the queries and
 * lcs_bvh_export return LCS_ERR_INVALID on a non-empty tree that no lcs_bvh_construct has built yet. */
LCS_API int lcs_bvh_update_leaves(lcs_bvh* h, const float* thickness, const float* x0, const float* x1,
                          const uint32_t* elems, lcs_stream stream);

/* LBVH::refit (lbvh.cpp:1038-1045): the inner boxes as unions of their children's, bit for bit the
 * reference's bottom-up walk (computed from each inner node's range of leaves in the walk's union order,
 * without a serial climb; the ranges are tables lcs_bvh_construct derives from the topology it builds). */
LCS_API int lcs_bvh_refit(lcs_bvh* h, lcs_stream stream);

/* update_*_tree_leave_aabb + refit in one launch (no reference counterpart as one call). */
LCS_API int lcs_bvh_update_refit(lcs_bvh* h, const float* thickness, const float* x0, const float* x1,
                         const uint32_t* elems, lcs_stream stream);

/* LBVH::broad_phase_query_from_verts (lbvh.cpp:1146-1167): every vertex box [x0,x1] +-
 * (thickness + d_hat) against a FACE tree; appends (vid, fid) to pairs (uint2) and adds the
 * number found to *d_count (device; the caller resets it).  Pairs beyond `capacity` are
 * counted but not written (the reference writes one pair past the end, lbvh.cpp:329-334). */
LCS_API int lcs_bvh_query_vf(const lcs_bvh* face_tree, const float* x0, const float* x1, uint32_t n_verts,
                     const float* d_hat, const float* thickness, uint32_t* pairs, uint32_t capacity,
                     uint32_t* d_count, lcs_stream stream);

/* LBVH::broad_phase_query_from_edges (lbvh.cpp:1168-1192): every edge's swept box +-
 * (thickness + d_hat of its first vertex) against an EDGE tree; keeps eid < adj_eid. */
LCS_API int lcs_bvh_query_ee(const lcs_bvh* edge_tree, const float* x0, const float* x1,
                     const uint32_t* edges, uint32_t n_edges, const float* d_hat,
                     const float* thickness, uint32_t* pairs, uint32_t capacity, uint32_t* d_count,
                     lcs_stream stream);

/* The candidate set of lcs_bvh_query_ee over every edge of the tree with thickness 0 and the same
 * d_hat for every edge's first vertex (no counterpart in the reference; what the Newton loop uses
 * when its scene satisfies that): each pair is met once, from the leaf with the lower Morton
 * position, and decided by the reference's test in the reference's direction, so the list holds the
 * same (eid, adj_eid) pairs, eid < adj_eid, in another order.  The edge tree must have been refitted
 * by this library (its node records carry the subtrees' last sorted positions). */
LCS_API int lcs_bvh_query_ee_sym(const lcs_bvh* edge_tree, const float* x0, const float* x1, const uint32_t* edges,
                                 float d_hat, uint32_t* pairs, uint32_t capacity, uint32_t* d_count,
                                 lcs_stream stream);

/* LBVH::check_health (lbvh.cpp:1033-1036).  Synchronises `stream`. host out. */
/* Candidate filter (no counterpart in the reference): the pairs of a VF (is_ee = 0, elems = faces)
 * or EE (is_ee = 1, elems = edges) candidate list whose boxes overlap at positions x, with the
 * boxes and the strict test of the queries above (query box +- thickness + d_hat of its first
 * vertex, leaf box +- thickness of its element's first vertex).  Applied to a swept-box list of a
 * tree it yields exactly the static-box list of the same tree at any x on the sweep, provided the
 * swept traversal did not end early.  Counts pairs beyond out_capacity without writing them. */
LCS_API int lcs_candidates_filter(int is_ee, const uint32_t* in_pairs, const uint32_t* in_count,
                                  uint32_t in_capacity, const float* x, const uint32_t* elems, const float* d_hat,
                                  const float* thickness, uint32_t* out_pairs, uint32_t out_capacity,
                                  uint32_t* out_count, lcs_stream stream);

LCS_API int lcs_bvh_health(lcs_bvh* h, int* healthy, lcs_stream stream);
/* fn_check_construction (lbvh.cpp:598-611), which lcs_bvh_construct runs after every build, run again on the
 * tree as it is now: the healthy flag is set, then cleared when an inner node's child does not name it as
 * its parent (or names a node outside the tree).  Read the flag with lcs_bvh_health. */
LCS_API int lcs_bvh_check_construction(lcs_bvh* h, lcs_stream stream);

/* Device buffers of the tree in the reference's LbvhData layout (lbvh.h:79-152: sa_parrent, sa_children,
 * sa_morton_sorted, sa_sorted_get_original, sa_is_healthy), valid until the handle is destroyed.  A caller
 * that writes into them must run lcs_bvh_check_construction before any refit or query.  Refit and queries
 * follow the topology of the last lcs_bvh_construct (its traversal records and refit tables), not edits
 * made here; rebuild to change the topology. */
typedef struct lcs_bvh_data_view {
    uint32_t n_leaves;
    uint32_t* parent;              /* 2 n - 1 */
    uint32_t* children;            /* 2 (2 n - 1): uint2 per node */
    uint64_t* morton_sorted;       /* n */
    uint32_t* sorted_get_original; /* n */
    uint32_t* is_healthy;          /* 1 */
} lcs_bvh_data_view;
LCS_API int lcs_bvh_data(const lcs_bvh* h, lcs_bvh_data_view* out);

/* Copies the tree out in the reference's LbvhData layout (lbvh.h:79-152), for tests and
 * interop; any pointer may be NULL.  node_aabb: 8 floats per node {min.xyz, 0, max.xyz, 0};
 * children: uint2 per node (leaves: (elem, elem)); parent[0] = 0xFFFFFFFF. */
LCS_API int lcs_bvh_export(const lcs_bvh* h, uint32_t* parent, uint32_t* children, uint32_t* object_idx,
                   uint64_t* morton, uint64_t* morton_sorted, uint32_t* sorted_get_original,
                   float* node_aabb, float* global_aabb6, lcs_stream stream);
LCS_API uint32_t lcs_bvh_num_leaves(const lcs_bvh* h);

/* ------------------------------------------------------------------------------------------
 * Forest of per-scene LBVHs (batched solver; no counterpart in the reference, which holds one
 * LBVH per tree kind).  Scenes are concatenated: element e of scene s is global element
 * elem_offsets[s] + e and refers to global vertex ids.  Each scene's tree is bit-identical to
 * the lcs_bvh tree of that scene alone (same global-AABB cover rule, Morton codes, sort order,
 * Karras topology over local element ids, refit boxes and query results).  Every scene needs at
 * least two elements.
 * ------------------------------------------------------------------------------------------ */
typedef struct lcs_forest lcs_forest;
/* elem_offsets / vert_offsets: host arrays of n_scenes + 1 prefix offsets (elem_offsets[0] = 0);
 * kind LCS_TREE_EDGE or LCS_TREE_FACE. */
LCS_API int lcs_forest_create(int kind, uint32_t n_scenes, const uint32_t* elem_offsets,
                              const uint32_t* vert_offsets, lcs_forest** out);
LCS_API int lcs_forest_destroy(lcs_forest* f);
/* reduce_*_tree_aabb + construct_tree for every scene in one set of launches */
LCS_API int lcs_forest_build(lcs_forest* f, const float* x, const uint32_t* elems, lcs_stream stream);
/* update_*_tree_leave_aabb + refit for every scene; this, the queries and lcs_forest_export_scene return
 * LCS_ERR_INVALID before the first lcs_forest_build */
LCS_API int lcs_forest_update_refit(lcs_forest* f, const float* thickness, const float* x0, const float* x1,
                                    const uint32_t* elems, lcs_stream stream);
/* broad_phase_query_from_verts for all scenes: vertex v queries the tree of vert_scene[v] */
LCS_API int lcs_forest_query_vf(const lcs_forest* face_forest, const float* x0, const float* x1,
                                uint32_t n_verts, const uint32_t* vert_scene, const float* d_hat,
                                const float* thickness, uint32_t* pairs, uint32_t capacity,
                                uint32_t* d_count, lcs_stream stream);
/* broad_phase_query_from_edges for all scenes (the forest's own edges are the queries) */
LCS_API int lcs_forest_query_ee(const lcs_forest* edge_forest, const float* x0, const float* x1,
                                const uint32_t* edges, const float* d_hat, const float* thickness,
                                uint32_t* pairs, uint32_t capacity, uint32_t* d_count, lcs_stream stream);
LCS_API int lcs_forest_health(lcs_forest* f, int* healthy, lcs_stream stream);
/* The queries' launch shape, tuned on a forest's first query (threads per block: 64, 128 or 256, each timed
 * once on that query, the fastest kept) and the tuned query's time in ms; 0 before the first query. */
LCS_API int lcs_forest_query_tuning(const lcs_forest* f, uint32_t* threads_per_block, float* query_ms);
/* one scene's tree in the layout of lcs_bvh_export (local node and element ids) */
LCS_API int lcs_forest_export_scene(const lcs_forest* f, uint32_t scene, uint32_t* parent, uint32_t* children,
                                    uint32_t* object_idx, uint64_t* morton_sorted,
                                    uint32_t* sorted_get_original, float* node_aabb, float* global_aabb6,
                                    lcs_stream stream);

/* ------------------------------------------------------------------------------------------
 * Narrow phase  (replaces NarrowPhasesDetector, Solver/CollisionDetector/narrow_phase.h:54-201)
 * Pair lists are the broad phase's uint2 lists; *d_count (device) holds how many are valid and
 * at most `capacity` of them are read.
 * ------------------------------------------------------------------------------------------ */

/* NarrowPhasesDetector::vf_ccd_query (narrow_phase.cpp:293-436, 609-676): ACCD on every
 * (vid, fid) candidate; d_toi[0] becomes min(d_toi[0], toi / 1.25) (the caller initialises it
 * to 1.0, as fn_reset_toi does).  toi_per_pair (optional) receives each pair's toi. */
LCS_API int lcs_ccd_vf(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x0,
               const float* x1, const uint32_t* faces, const uint32_t* body, const float* offset,
               float* d_toi, float* toi_per_pair, int flags, lcs_stream stream);

/* NarrowPhasesDetector::ee_ccd_query (narrow_phase.cpp:438-593, 678-740). */
LCS_API int lcs_ccd_ee(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x0,
               const float* x1, const uint32_t* edges, const uint32_t* body, const float* offset,
               float* d_toi, float* toi_per_pair, int flags, lcs_stream stream);
/* Batched scenes (no counterpart in the reference): the VF (is_ee = 0, elems = faces) or EE
 * (is_ee = 1, elems = edges) step bound of every candidate, lowered into the bound of the pair's
 * own scene, d_toi_per_scene[vert_scene[first vertex]] (each initialised to 1 by the caller). */
LCS_API int lcs_ccd_batch(int is_ee, const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity,
                          const float* x0, const float* x1, const uint32_t* elems, const uint32_t* body,
                          const float* offset, const uint32_t* vert_scene, float* d_toi_per_scene,
                          float* toi_per_pair, int flags, lcs_stream stream);

/* NarrowPhasesDetector::vf_dcd_query_repulsion (narrow_phase.cpp:771-933, 1102-1170): barrier
 * contact pairs with d^2 < (offset + d_hat)^2; appended to out, count added to *d_out_count. */
LCS_API int lcs_dcd_vf(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x,
               const uint32_t* faces, const uint32_t* body, const float* vert_area,
               const float* face_area, const float* d_hat, const float* offset, float kappa,
               lcs_pair* out, uint32_t out_capacity, uint32_t* d_out_count, lcs_stream stream);

/* NarrowPhasesDetector::ee_dcd_query_repulsion (narrow_phase.cpp:935-1098, 1171-1249). */
LCS_API int lcs_dcd_ee(const uint32_t* pairs, const uint32_t* d_count, uint32_t capacity, const float* x,
               const uint32_t* edges, const uint32_t* body, const float* edge_area,
               const float* d_hat, const float* offset, float kappa, lcs_pair* out,
               uint32_t out_capacity, uint32_t* d_out_count, lcs_stream stream);

/* NarrowPhasesDetector::device_perPair_evaluate_gradient_hessian (narrow_phase.cpp:2550-2676,
 * 2817-2843): b[v] += k1 w_v n and diag[v] += k2 w_v^2 n n^T for every pair (soft vertices). */
LCS_API int lcs_contact_grad_diag(const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity,
                          float* b, float* diag, lcs_stream stream);

/* Affine bodies (ABD).  A body's 12 DOFs q = [p, a0, a1, a2] are four DOF-slot rows of the system
 * (vertex ids body_dof[b] .. body_dof[b] + 3); its mesh vertices move by x = p + A x_bar. */
typedef struct lcs_abd_view {
    const uint32_t* body;      /* per vertex: affine-body id, 0xFFFFFFFF = soft */
    const float* model_x;      /* float4 per vertex: body-frame rest position x_bar of rigid vertices */
    const uint32_t* body_dof;  /* per body: vertex id of its first DOF slot */
} lcs_abd_view;
/* lcs_contact_grad_diag with the ABD remap (collision_data.h:198-268, narrow_phase.cpp:2598-2676): a rigid
 * side of a pair adds to its body's four DOF slots with weights sum_i w_i (1, x_bar_i). */
LCS_API int lcs_contact_grad_diag_abd(const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity, float* b,
                                      float* diag, const lcs_abd_view* abd, lcs_stream stream);

/* NarrowPhasesDetector::compute_contact_energy_from_iter_start_list + download_energy
 * (narrow_phase.cpp:2968-3070, 123-130): sum of kappa * area * barrier over the pairs at
 * positions x, accumulated in FP64 into *d_energy (device double, caller resets). */
LCS_API int lcs_contact_energy(const lcs_pair* pairs, const uint32_t* d_count, uint32_t capacity,
                       const float* x, const float* d_hat, const float* offset, double* d_energy,
                       lcs_stream stream);

/* Contact off-diagonal blocks: the per-vertex adjacency + two-level triplet sort + assembly
 * (prescan_pervert_adj_list, construct_pervert_adj_list, device_sort_contact_triplet,
 * device_assemble_contact_triplet; narrow_phase.cpp:1264-1426, 1434-2362) as one device radix
 * sort of (row, col) keys and a segmented sum.  The assembler owns the output BSR. */
typedef struct lcs_assembler lcs_assembler;
LCS_API int lcs_assembler_create(uint32_t n_rows, uint32_t pair_capacity, lcs_assembler** out);
LCS_API int lcs_assembler_destroy(lcs_assembler* a);
LCS_API int lcs_contact_offdiag_bsr(lcs_assembler* a, const lcs_pair* pairs, const uint32_t* d_count,
                            uint32_t capacity, lcs_stream stream);
/* An assembler sized for pairs with rigid sides (up to 8 generalised DOFs, 56 blocks per pair), and the
 * off-diagonal blocks with the ABD remap (fn_assemble_triplet_sorted, narrow_phase.cpp:1760-1880). */
LCS_API int lcs_assembler_create_abd(uint32_t n_rows, uint32_t pair_capacity, lcs_assembler** out);
LCS_API int lcs_contact_offdiag_bsr_abd(lcs_assembler* a, const lcs_pair* pairs, const uint32_t* d_count,
                                        uint32_t capacity, const lcs_abd_view* abd, lcs_stream stream);
/* Device pointers of the assembled BSR; *d_nnzb is a device uint32. */
LCS_API int lcs_assembler_bsr(const lcs_assembler* a, lcs_bsr* out, const uint32_t** d_nnzb);
/* NarrowPhasesDetector::download_contact_triplet (narrow_phase.cpp:207-233): copies the BSR
 * into caller device buffers (at most max_blocks blocks) and returns the block count in
 * *nnzb (host).  Synchronises `stream`. */
LCS_API int lcs_assembler_export(const lcs_assembler* a, uint32_t* row_ptr, uint32_t* col, float* val,
                                 uint32_t max_blocks, uint32_t* nnzb, lcs_stream stream);

/* ------------------------------------------------------------------------------------------
 * SpMV + Jacobi PCG  (replaces ConjugateGradientSolver, Solver/LinearSolver/precond_cg.h:17-71,
 * and NewtonSolver::device_SpMV, Solver/SimulationSolver/newton_solver.cpp:3397-3427)
 * ------------------------------------------------------------------------------------------ */

/* y = D x + A x + B x (A, B may be NULL): fn_pcg_spmv_diag + fn_pcg_spmv_offdiag_block_rbk on the
 * material and the contact triplets (newton_solver.cpp:259-270, 347-472). */
LCS_API int lcs_spmv(uint32_t n, const float* diag, const lcs_bsr* A, const lcs_bsr* B, const float* x,
             float* y, lcs_stream stream);

enum {
    LCS_PCG_FP64_DOTS = 1, /* precision form: FP64 dot products and residual reductions */
    LCS_PCG_PLAIN = 2,     /* reference dispatch structure: one kernel per op, host check */
    LCS_PCG_NO_STATS = 4,  /* fused path: do not synchronise to fill *stats */
    LCS_PCG_ROWS = 8,      /* row-resident persistent solve (one thread per block row, state in registers);
                              falls back to the persistent solve when the rows exceed one thread each */
    LCS_PCG_SINGLE_REDUCTION = 16 /* with LCS_PCG_ROWS: the single-reduction (Chronopoulos-Gear) form of the
                              same PCG, r.u and (A u).u summed in one grid reduction: two grid-wide
                              synchronisations per iteration instead of three; the same Krylov iterates in
                              exact arithmetic, rounding as stable as the classic form */
};

typedef struct lcs_pcg_opts {
    int32_t max_iter;    /* pcg_iter_count (reference default 100) */
    float rel_tol;       /* stop when ||r|| <= rel_tol * ||r0|| (<= 0: off) */
    float abs_rz_tol;    /* stop when r.z < abs_rz_tol (reference: 1e-10) */
    int32_t check_every; /* reference: 25 */
    int32_t flags;
} lcs_pcg_opts;

typedef struct lcs_pcg_stats {
    int32_t iterations;
    float rel_residual; /* ||r|| / ||r0|| at the last check */
    float dot_rz;
    int32_t status;     /* lcs_status of the solve (NaN -> LCS_ERR_NAN) */
} lcs_pcg_stats;

typedef struct lcs_pcg lcs_pcg;
LCS_API int lcs_pcg_create(uint32_t n, lcs_pcg** out);
LCS_API int lcs_pcg_destroy(lcs_pcg* p);
/* ConjugateGradientSolver::device_solve (precond_cg.cpp:626-771): x = A^-1 b with x0 = 0.
 * stats (host, may be NULL) is filled after the solve (synchronises the stream unless
 * LCS_PCG_NO_STATS).  Device copy of the stats: lcs_pcg_device_stats. */
LCS_API int lcs_pcg_solve(lcs_pcg* p, const float* diag, const lcs_bsr* A, const lcs_bsr* B,
                  const float* b, float* x, const lcs_pcg_opts* opts, lcs_pcg_stats* stats,
                  lcs_stream stream);
LCS_API const lcs_pcg_stats* lcs_pcg_device_stats(const lcs_pcg* p);
/* Test hook for failure detection (no counterpart in the reference, whose bounded wait is wait_for_write,
 * lbvh.cpp:62-82): runs the slice-resident solve's reduction barrier (which = 0) or its neighbour-flag wait
 * (which = 1) on `blocks` (2..32) co-resident blocks, each waiting for all others, with block missing_block
 * (-1: none) never arriving or publishing.  Every wait gives up after spin_limit polls (1..2^24; the solves use
 * 2^24).  Returns LCS_ERR_TIMEOUT when a wait ran out, LCS_OK when all completed.  No block waits forever and
 * the context stays usable. */
LCS_API int lcs_debug_pcg_wait(int32_t which, int32_t missing_block, uint32_t blocks, uint32_t spin_limit,
                               lcs_stream stream);

/* Allocation-free variant of lcs_pcg_solve (fused solve only); it has no counterpart in the
 * reference.  For callers that cannot allocate device memory while they run: cudaMalloc and
 * cudaFree synchronise the whole device, which a fixed-latency loop cannot afford, and a host
 * that gives all device memory to its own pool allocator leaves none to allocate.  Needs no
 * handle: the working vectors live in one static device array (7.3 MB per GPU).  Under CUDA's
 * default lazy module loading that array is reserved on a device the first time the library's
 * PCG module is used there -- the first call of this function or the first launch of any PCG
 * solve -- and kept until the process exits; make one call on each device before a pool takes
 * its memory (if the memory is gone, the set-up fails with LCS_ERR_CAPACITY).  At most 65,536
 * block rows (larger systems: LCS_ERR_CAPACITY).  Calls on one device share that array, so
 * calls whose work overlaps on the GPU race and must be ordered by the caller.  The first call
 * on each device does a one-time set-up (it looks up the array's device address and caches it
 * for the process); make it before any stream capture, and do not call this function on a
 * device after cudaDeviceReset.  opts NULL: the defaults of lcs_pcg_solve (100 iterations,
 * rel 1e-4, r.z 1e-10, checked every 25).  LCS_PCG_PLAIN, LCS_PCG_ROWS and
 * LCS_PCG_SINGLE_REDUCTION are rejected (LCS_ERR_INVALID). */
LCS_API int lcs_pcg_solve_noalloc(uint32_t n, const float* diag, const lcs_bsr* A, const lcs_bsr* B,
                                  const float* b, float* x, const lcs_pcg_opts* opts, lcs_pcg_stats* stats,
                                  lcs_stream stream);

/* Batched scenes (no counterpart in the reference): n_scenes independent systems, scene s owning
 * block rows [row_offsets[s], row_offsets[s+1]) of one BSR pair (row_offsets: device array of
 * n_scenes + 1; host_row_offsets: the same offsets in host memory), solved in one launch with one
 * thread-block cluster of `cluster` CTAs (1, 2, 4, 8 or 16) per scene, or with `cluster` = 0 one
 * cluster per scene of the smallest size that leaves it at most T chunks of 256 rows per CTA (one
 * launch per size, side by side on streams forked from `stream`).  T is tuned by the first such call
 * on the handle: it solves the system once for each T in {2, 4, 8, 16}, times each on `stream`
 * (synchronising it) and keeps the fastest for later calls (lcs_pcg_batch_tuning reports it).
 * Each scene has its own
 * alpha, beta and stop decision (the rules of lcs_pcg_solve); its result does not depend on
 * `cluster` or on the other scenes.  active: device flags per scene (0: skip, x = 0) or NULL.
 * stats_per_scene: device array of n_scenes.  Asynchronous; the handle must hold at least
 * host_row_offsets[n_scenes] rows. */
LCS_API int lcs_pcg_solve_batch(lcs_pcg* p, uint32_t n_scenes, const uint32_t* row_offsets,
                                const uint32_t* host_row_offsets, const uint32_t* active, const float* diag,
                                const lcs_bsr* A, const lcs_bsr* B, const float* b, float* x,
                                const lcs_pcg_opts* opts, lcs_pcg_stats* stats_per_scene, int cluster,
                                lcs_stream stream);
/* The chunks-per-CTA target the batched solve tuned (0 before the first cluster = 0 call) and its
 * measured solve time in ms. */
LCS_API int lcs_pcg_batch_tuning(const lcs_pcg* p, uint32_t* chunks_per_cta, float* solve_ms);

/* ------------------------------------------------------------------------------------------
 * Cloth energies  (replaces the evaluate kernels of NewtonSolver::compile_evaluate,
 * Solver/SimulationSolver/newton_solver.cpp:1002-1175, and the elastic energy of the line
 * search, Solver/SimulationSolver/solver_interface.cpp:505-728)
 *
 * Per-element outputs use the reference's layouts: gradients one float4 per (element, local
 * vertex); Hessians one float3x3 record (three float4 columns) per block, the N diagonal blocks
 * first, then the off-diagonal blocks (i, j), i != j, in row-major order (row vertex i, column
 * vertex j): N*N blocks per element.
 * ------------------------------------------------------------------------------------------ */
/* ConstitutiveStretchModelCloth / ConstitutiveBendingModelCloth (physical_material.h:11-23) */
enum { LCS_STRETCH_SPRING = 0, LCS_STRETCH_BW98 = 1 };
enum { LCS_BENDING_NONE = 0, LCS_BENDING_QUADRATIC = 1, LCS_BENDING_DIHEDRAL = 2 };

/* fn_evaluate_spring (newton_solver.cpp:1002-1050): edges uint2, per-spring rest length and
 * stiffness; 2 gradients and 4 blocks ((0,0) (1,1) (0,1) (1,0)) per spring. */
LCS_API int lcs_eval_springs(const float* x, const uint32_t* edges, const float* rest_len, const float* stiffness,
                             uint32_t n, float* gradients, float* hessians, lcs_stream stream);
/* fn_evaluate_stretch_face (newton_solver.cpp:1052-1100): Baraff-Witkin stretch + shear with
 * projected Hessians (stretch_energy.h:156-476).  faces uint4; dm_inv 4 floats per face (the rest
 * Dm^-1 columns, StretchEnergy::get_Dm_inv); rest_area; mu_lambda 2 floats per face. */
LCS_API int lcs_eval_stretch_faces(const float* x, const uint32_t* faces, const float* dm_inv, const float* rest_area,
                                   const float* mu_lambda, uint32_t n, float* gradients, float* hessians,
                                   lcs_stream stream);
/* fn_evaluate_bending (newton_solver.cpp:1102-1175): dihedral angle of the hinge (s.x, s.y) with
 * wings s.z, s.w; gradient k (theta - rest_angle) dtheta/dx, Gauss-Newton blocks k g_i g_j^T with
 * k = stiffness * scaling * rest_hbar (init_sim_data.cpp:420-448). */
LCS_API int lcs_eval_bending(const float* x, const uint32_t* stencils, const float* rest_angle, const float* rest_hbar,
                             const float* stiffness, float scaling, uint32_t n, float* gradients, float* hessians,
                             lcs_stream stream);

/* The per-element arrays of a cloth system (device pointers), as SimulationData holds them. */
typedef struct lcs_cloth_elements {
    uint32_t n_verts, n_springs, n_stretch_faces, n_bending;
    const float* mass;                 /* per vertex */
    const uint8_t* is_fixed;           /* per vertex, or NULL */
    const uint32_t* springs;           /* uint2 */
    const float* spring_rest_len;
    const float* spring_stiffness;
    const uint32_t* stretch_faces;     /* uint4 */
    const float* stretch_dm_inv;       /* 4 floats per face */
    const float* stretch_area;
    const float* stretch_mu_lambda;    /* 2 floats per face */
    const uint32_t* bending_edges;     /* uint4 stencils */
    const float* bending_rest_angle;
    const float* bending_hbar;
    const float* bending_stiffness;
    float bending_scaling;             /* stiffness_bending_ui */
} lcs_cloth_elements;
/* SolverInterface::device_compute_elastic_energy without the ground term: writes 4 doubles
 * (device) -- inertia (with the Dirichlet factor on fixed vertices), springs, stretch faces,
 * bending -- each summed in FP64.  Asynchronous. */
LCS_API int lcs_material_energy(const lcs_cloth_elements* m, const float* x, const float* x_tilde, float dt,
                                float stiffness_dirichlet, double* energy, lcs_stream stream);

/* ------------------------------------------------------------------------------------------
 * Newton loop  (replaces NewtonSolver::physics_step_GPU and its contact glue,
 * Solver/SimulationSolver/newton_solver.cpp:3174-3375, 3685-3884, 4051-4345)
 * ------------------------------------------------------------------------------------------ */
typedef struct lcs_scene_desc {
    uint32_t n_verts, n_faces, n_edges, n_bending;
    const float* x;             /* host float4 per vertex: rest = initial positions */
    const float* v;             /* host float4 per vertex, or NULL (at rest) */
    const uint32_t* faces;      /* host uint4 */
    const uint32_t* edges;      /* host uint2 (springs and the edge tree) */
    const uint32_t* bending;    /* host uint4 stencils (e0, e1, opposite of face 0, of face 1) */
    const float* bending_Q;     /* host 16 floats per stencil (init_sim_data.cpp:455-480) */
    const float* rest_len;      /* host, per edge */
    const float* vert_area;     /* host, per vertex (init_mesh_data.cpp:780-870) */
    const float* face_area;
    const float* edge_area;
    const float* mass;          /* host, per vertex */
    const float* d_hat;         /* host, per vertex (init_collision_data.cpp:67-171) */
    const float* offset;        /* host, per vertex */
    const uint32_t* body;       /* host affine-body id per vertex, or NULL (all soft) */
    const uint8_t* pinned;      /* host, or NULL */
    const int8_t* anim_group;   /* host, per vertex animation group of pinned vertices (-1 none) */
    uint32_t n_anim;
    const float* anim;          /* host, 16 floats per group (FixedPointAnimationInfo): centre xyz, unit axis xyz,
                                   rad/s, mode (bits: 1 rotate, 2 scale, 4 translate), translation velocity xyz,
                                   scale rate xyz, 2 pad */
    float dt;
    float gravity[3];
    float kappa;                /* stiffness_collision */
    float spring_k;             /* stiffness_spring */
    float bending_k;            /* area_bending_stiffness */
    float dirichlet;            /* stiffness_dirichlet */
    float damping;              /* damping_cloth */
    int32_t use_floor;
    float floor_y;
    int32_t nonlinear_iters;    /* nonlinear_iter_count */
    int32_t pcg_max_iter;       /* pcg_iter_count */
    float pcg_rel_tol;
    float pcg_abs_rz_tol;
    int32_t pcg_check_every;    /* host check cadence of the plain loop (reference: 25) */
    /* cloth models (ClothMaterial, physical_material.h:53-62; element culling init_sim_data.cpp:205-270).
     * stretch_model LCS_STRETCH_SPRING: springs on `edges` with rest_len and spring_k;
     * LCS_STRETCH_BW98: the stretch faces below.  bending_model LCS_BENDING_DIHEDRAL: the stencils
     * in `bending` with bending_rest_angle / bending_hbar, stiffness bending_k * bending_scaling * hbar;
     * LCS_BENDING_QUADRATIC: the rest-relative quadratic form with bending_Q and bending_k (the
     * reference's disabled branch, newton_solver.cpp:3013-3045); LCS_BENDING_NONE: no bending. */
    int32_t stretch_model;
    int32_t bending_model;
    uint32_t n_stretch_faces;
    const uint32_t* stretch_faces;   /* host uint4, faces with a free vertex */
    const float* stretch_dm_inv;     /* host, 4 floats per stretch face (rest Dm^-1 columns) */
    const float* stretch_area;       /* host, rest area per stretch face */
    float stretch_mu, stretch_lambda;/* thickness-scaled Lame parameters (init_sim_data.cpp:388-397) */
    const float* bending_rest_angle; /* host, per stencil */
    const float* bending_hbar;       /* host, per stencil: (A0 + A1) / (3 |e|) */
    float bending_scaling;           /* stiffness_bending_ui */
    /* affine bodies (ABD; init_sim_data.cpp:520-757).  Body b's DOFs q = [p, a0, a1, a2] are the four
     * vertex records body_dof[b] .. body_dof[b] + 3 of x / v (slots in no face or edge, d_hat < 0 so that
     * they query nothing); its mesh vertices carry `body` = b and their body-frame positions in model_x. */
    uint32_t n_bodies;
    const uint32_t* body_dof;        /* host, per body */
    const float* body_mass;          /* host, 16 floats per body: the 4 x 4 mass matrix [M, MI^T; MI, I] */
    const float* body_volume;        /* host, per body */
    const float* body_kappa;         /* host, per body: RigidMaterial stiffness (orthogonality) */
    const float* model_x;            /* host float4 per vertex (rigid vertices; others ignored) */
    /* per-element material parameters (SimulationData's sa_stretch_faces_mu_lambda,
     * sa_bending_edges_stiffness, sa_stretch_spring_stiffness), or NULL for the scalars above */
    const float* stretch_mu_lambda;  /* host, 2 floats per stretch face */
    const float* bending_stiffness;  /* host, per stencil (area_bending_stiffness of its mesh) */
    const float* spring_stiffness;   /* host, per edge */
} lcs_scene_desc;

enum {
    LCS_NEWTON_PLAIN = 1,   /* the reference's dispatch structure (one-scene comparator) */
    LCS_NEWTON_FP64 = 2,    /* precision form: FP64 PCG reductions, ACCD step bound in FP64 */
    LCS_NEWTON_PROFILE = 4, /* per-phase CUDA-event timing (lcs_newton_profile) */
    LCS_NEWTON_PCG_SINGLE_REDUCTION = 8, /* fused mode: single-reduction row-resident PCG (LCS_PCG_SINGLE_REDUCTION) */
    LCS_NEWTON_FULL_TRAVERSAL = 16, /* fused mode: every candidate list by a traversal (no DCD filtering of the
                                      previous iteration's CCD lists) */
    LCS_NEWTON_ENERGY_LINESEARCH = 32, /* use_energy_linesearch (scene_params.h:41): after the CCD bound, halve the
                                         step until the energy (inertia, cloth, barrier of the iteration-start
                                         pairs; FP64 sums) decreases (newton_solver.cpp:3790-3834).  Single scenes;
                                         the fused loop evaluates 7 step lengths per launch and decides on the
                                         device, the plain loop one per host round trip as the reference does. */
    LCS_NEWTON_PCG_GLOBAL_MATRIX = 64, /* with LCS_NEWTON_PCG_SINGLE_REDUCTION: read the material matrix from
                                         global memory every iteration (the grid of 256-row blocks) instead of
                                         the slice-resident solve (one block per SM, its rows' leading matrix
                                         groups held in shared memory), which is used where the rows fit */
    LCS_NEWTON_DETERMINISTIC = 128 /* sums without atomics: the cloth terms are evaluated per element and summed
                                      per row and per block in element order, the contact pairs are sorted into a
                                      canonical order (by type and vertex indices) before their gradient,
                                      diagonal and off-diagonal blocks are summed in that order.  A scene's step
                                      is then bit-identical from run to run and, in a batch, whatever the other
                                      scenes are.  The reference accumulates with atomics (narrow_phase.cpp:
                                      2550-2676, newton_solver.cpp:705-814); this flag has no counterpart
                                      there.  Not with affine bodies or the energy line search; scenes below
                                      2^21 vertices. */
};

typedef struct lcs_newton_stats {
    int32_t newton_iters;
    int32_t pcg_iters;
    float last_toi;
    float last_rel_residual;
    uint32_t vf_candidates, ee_candidates, contact_pairs, ccd_vf_candidates, ccd_ee_candidates;
    int32_t status;
    int32_t retries;  /* iterations re-run after a buffer grew */
    float host_ms;    /* host wall time of the step */
    float last_alpha; /* step length of the last iteration (the CCD bound, or the line search's choice) */
    int32_t ls_halvings; /* step halvings of the energy line search in this step */
} lcs_newton_stats;

/* One Newton iteration of the last step: the figures NewtonSolver::line_search logs per iteration
 * (newton_solver.cpp:3770-3780; PCG iterations and error, precond_cg.cpp:763-768) and the iteration's
 * direction norm (the small-step test, newton_solver.cpp:3784-3800). */
typedef struct lcs_newton_iter_record {
    int32_t pcg_iters;
    float rel_residual; /* |r| / |r0| where the solve stopped */
    float toi;          /* CCD step bound */
    float max_dx;       /* max over the solve's unknowns of |dx| */
    uint32_t vf_candidates, ee_candidates, contact_pairs, ccd_vf_candidates, ccd_ee_candidates;
} lcs_newton_iter_record;

typedef struct lcs_newton lcs_newton;
/* NewtonSolver::init_solver (newton_solver.h:31-51): uploads the scene, builds the material
 * block pattern, allocates the contact buffers (CollisionData sizing, collision_data.h:445-485).
 * stream: the stream all work of this solver goes to (NULL: the solver creates one). */
LCS_API int lcs_newton_create(const lcs_scene_desc* desc, int flags, lcs_stream stream, lcs_newton** out);
/* Batched scenes (no counterpart in the reference): n_scenes independent scenes stepped
 * together, one set of launches per Newton phase for all of them (forests of per-scene LBVHs,
 * per-scene step bounds, per-scene PCG on thread-block clusters of pcg_cluster CTAs: 1, 2, 4, 8
 * or 16, or 0 to size the clusters from the largest scene).  Every scene runs its own Newton loop (its own small-step and Dirichlet tests); a scene
 * that has finished is switched off for the rest of the step.  The scenes must share dt,
 * gravity, stiffnesses and solver settings and run with the floor off; LCS_NEWTON_PLAIN is
 * rejected.  A scene's trajectory does not depend on the other scenes of the batch (up to the
 * summation order of atomic accumulations). */
LCS_API int lcs_newton_create_batch(const lcs_scene_desc* descs, uint32_t n_scenes, int flags, lcs_stream stream,
                                    int pcg_cluster, lcs_newton** out);
LCS_API uint32_t lcs_newton_num_scenes(const lcs_newton* h);
/* per-scene figures of the last step: newton_iters, pcg_iters, last_toi, last_rel_residual */
LCS_API int lcs_newton_scene_stats(const lcs_newton* h, uint32_t scene, lcs_newton_stats* stats);
/* one scene's x, v (float4 per vertex) to host memory; synchronises the solver's stream */
LCS_API int lcs_newton_download_scene(const lcs_newton* h, uint32_t scene, float* x_out, float* v_out);
LCS_API int lcs_newton_destroy(lcs_newton* h);
/* The last Newton iteration's start positions (sa_x_iter_start), direction (sa_cgX) and the step's
 * inertial target (sa_x_tilde), float4 per vertex, to host memory (any may be NULL); synchronises. */
LCS_API int lcs_newton_last_iterate(const lcs_newton* h, float* x_iter_out, float* dx_out, float* x_tilde_out);
/* NewtonSolver::physics_step_GPU (newton_solver.cpp:4051-4345) on the device-resident state. */
LCS_API int lcs_newton_step(lcs_newton* h, lcs_newton_stats* stats);
/* The same step with host positions / velocities in and out (float4 per vertex, any may be NULL). */
/* Per-iteration records of the last single-scene step (at most cap are written; *n_out = the number of
 * iterations the step ran).  A batch reports none (*n_out = 0). */
LCS_API int lcs_newton_iteration_log(const lcs_newton* h, lcs_newton_iter_record* out, int32_t cap, int32_t* n_out);
LCS_API int lcs_newton_step_host(lcs_newton* h, const float* x_in, const float* v_in, float* x_out, float* v_out,
                                 lcs_newton_stats* stats);
/* Copies the positions / velocities (float4 per vertex) to host buffers; either may be NULL.
 * Synchronises the solver's stream. */
LCS_API int lcs_newton_download(const lcs_newton* h, float* x_out, float* v_out);
/* Replaces the positions / velocities (float4 per vertex; either may be NULL) with host buffers, as
 * SolverInterface::load_saved_state_from_host (solver_interface.cpp:275-412) does before the next frame.
 * Synchronises the solver's stream. */
LCS_API int lcs_newton_upload(lcs_newton* h, const float* x_in, const float* v_in);
/* Device pointers of the solver's positions and velocities (float4 per vertex).  Positions written
 * through this pointer must be announced with lcs_newton_invalidate(h), so that the next step does not
 * reuse candidate lists of the old positions. */
LCS_API int lcs_newton_state(const lcs_newton* h, float** d_x, float** d_v);
/* The positions changed outside the solver (through lcs_newton_state): the next step traverses the
 * trees for its first DCD lists instead of filtering the previous step's CCD lists. */
LCS_API int lcs_newton_invalidate(lcs_newton* h);
/* Sets the frame counter (scene_params.h:79 current_frame, advanced once per step by app_simulation.cpp:134):
 * the next step animates the pinned vertices to time (frame + 1) * dt.  Used with lcs_newton_upload to
 * resume from a saved frame state. */
LCS_API int lcs_newton_set_frame(lcs_newton* h, uint32_t frame);
/* The number of steps taken since creation or the last lcs_newton_set_frame plus the frame set there. */
LCS_API int lcs_newton_get_frame(const lcs_newton* h, uint32_t* frame_out);
/* Accumulated per-phase GPU time (LCS_NEWTON_PROFILE): build, material, DCD broad, DCD narrow,
 * assembly, PCG, CCD broad, CCD narrow, apply -- and how many times each ran. */
LCS_API int lcs_newton_profile(const lcs_newton* h, double* phase_ms, int32_t* launches, int n);
LCS_API int lcs_newton_reset_profile(lcs_newton* h);
LCS_API int lcs_newton_counts(const lcs_newton* h, uint32_t* nnz_material, uint32_t* cap_vf, uint32_t* cap_ee,
                              uint32_t* cap_pairs);
/* Which PCG the Newton loop runs: 0 plain kernels, 1 persistent CSR solve, 2 row-resident,
 * 3 single-reduction row-resident, 4 single-reduction slice-resident (-1: null handle).  No counterpart in the reference. */
LCS_API int lcs_newton_pcg_kind(const lcs_newton* h);
/* A batch's tuned PCG shape (lcs_pcg_batch_tuning of its solver): chunks of 256 rows per CTA and the
 * tuned solve's time in ms; 0 before the first step of a batch created with pcg_cluster 0. */
LCS_API int lcs_newton_batch_tuning(const lcs_newton* h, uint32_t* chunks_per_cta, float* solve_ms);
/* A batch's tuned traversal shapes (lcs_forest_query_tuning of its face and edge forests): threads per block
 * of the VF and EE queries; 0 before the first step. */
LCS_API int lcs_newton_batch_query_tuning(const lcs_newton* h, uint32_t* vf_threads, uint32_t* ee_threads);

#ifdef __cplusplus
}
#endif
#endif /* LCS_GPU_H */
