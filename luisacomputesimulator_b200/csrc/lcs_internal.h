// lcs_internal.h -- error recording shared by the C-ABI entry points.
#pragma once
#include "../../include/lcs_gpu.h"

// Counts one kernel launch of this library (lcs_launch_count).
void lcs_count_launch();

// Records `msg` as this thread's last error and returns `code`.
int lcs_fail(int code, const char* msg);

// Row-resident PCG solve with the material matrix in SELL-32 (slices of 32 rows; slot k of a
// slice at col[32 * k + lane], value component c at val[(9 * k + c) * 32 + lane], k counted from
// slice_ptr[slice]) and the contact blocks in CSR.  LCS_ERR_CAPACITY if the rows do not fit.
int lcs_pcg_solve_sell(lcs_pcg* P, const float* diag, const uint32_t* slice_ptr, const uint32_t* col,
                       const float* val, const lcs_bsr* B, const float* b, float* x, const lcs_pcg_opts* opts,
                       lcs_pcg_stats* stats, lcs_stream stream);
// Most block rows the row-resident solve holds on the current device (one thread per row).
int64_t lcs_pcg_rows_capacity();

// construct_tree with the reference's host sort (Morton codes downloaded, sorted on the CPU,
// uploaded; lbvh.cpp:983-993) -- used by the plain one-scene comparator loop only.
int lcs_bvh_construct_host_sort(lcs_bvh* h, lcs_stream stream);

// lcs_bvh_query_vf / _ee that also OR 1 into *capped (device, may be NULL) when a traversal ends
// early (full stack or the 100000-step limit), i.e. when the list may be incomplete.
int lcs_bvh_query_vf_capped(const lcs_bvh* t, const float* x0, const float* x1, uint32_t n_verts, const float* d_hat,
                            const float* thickness, uint32_t* pairs, uint32_t capacity, uint32_t* d_count,
                            uint32_t* capped, lcs_stream stream);
int lcs_bvh_query_ee_capped(const lcs_bvh* t, const float* x0, const float* x1, const uint32_t* edges, uint32_t n_edges,
                            const float* d_hat, const float* thickness, uint32_t* pairs, uint32_t capacity,
                            uint32_t* d_count, uint32_t* capped, lcs_stream stream);
int lcs_forest_query_vf_capped(const lcs_forest* f, const float* x0, const float* x1, uint32_t n_verts,
                               const uint32_t* vert_scene, const float* d_hat, const float* thickness, uint32_t* pairs,
                               uint32_t capacity, uint32_t* d_count, uint32_t* capped, lcs_stream stream);
int lcs_forest_query_ee_capped(const lcs_forest* f, const float* x0, const float* x1, const uint32_t* edges,
                               const float* d_hat, const float* thickness, uint32_t* pairs, uint32_t capacity,
                               uint32_t* d_count, uint32_t* capped, lcs_stream stream);
