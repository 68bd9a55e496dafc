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
// c_ptr / c_col / c_val / c_ok (optional): the contact blocks B again in the same SELL-32 layout
// (lcs_contact_to_sell); the solve reads them instead of B's CSR while *c_ok is set on the device.
int lcs_pcg_solve_sell(lcs_pcg* P, const float* diag, const uint32_t* slice_ptr, const uint32_t* col,
                       const float* val, const lcs_bsr* B, const float* b, float* x, const lcs_pcg_opts* opts,
                       lcs_pcg_stats* stats, lcs_stream stream, const uint32_t* c_ptr = nullptr,
                       const uint32_t* c_col = nullptr, const float* c_val = nullptr, const int* c_ok = nullptr);
// The CSR matrix B (n block rows) rewritten as SELL-32 with 4-slot groups (the layout lcs_pcg_solve_sell
// takes for the material matrix): width (ceil(n / 32) words of scratch), ptr (ceil(n / 32) + 1 slot
// offsets), col (32 words per slot), val (288 floats per slot).  *ok (device) is set to 0 when the
// slots would exceed cap_slots, and nothing else is written then.
int lcs_contact_to_sell(uint32_t n, const lcs_bsr* B, uint32_t* width, uint32_t* ptr, uint32_t* col, float* val,
                        uint32_t cap_slots, int* ok, lcs_stream stream);
// Most block rows the row-resident solve holds on the current device (one thread per row).
int64_t lcs_pcg_rows_capacity();
// lcs_pcg_opts flag: keep the SELL matrix in global memory (k_pcg_cg1) where the slice-resident
// single-reduction solve (one block per SM, matrix groups in shared memory) would apply.
constexpr int LCS_PCG_INTERNAL_NO_RESIDENT = 1 << 16;
// 1 if single-reduction SELL solves of this handle run slice-resident (k_pcg_res), else 0.
int lcs_pcg_resident(lcs_pcg* P);

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
int lcs_bvh_query_ee_sym_capped(const lcs_bvh* t, const float* x0, const float* x1, const uint32_t* edges,
                                float d_hat, uint32_t* pairs, uint32_t capacity, uint32_t* d_count, uint32_t* capped,
                                lcs_stream stream);
// only (optional): a per-vertex mask; queries whose (first) vertex is not set are skipped.
int lcs_forest_query_vf_capped(const lcs_forest* f, const float* x0, const float* x1, uint32_t n_verts,
                               const uint32_t* vert_scene, const float* d_hat, const float* thickness, uint32_t* pairs,
                               uint32_t capacity, uint32_t* d_count, uint32_t* capped, lcs_stream stream,
                               const uint8_t* only = nullptr);
int lcs_forest_query_ee_capped(const lcs_forest* f, const float* x0, const float* x1, const uint32_t* edges,
                               const float* d_hat, const float* thickness, uint32_t* pairs, uint32_t capacity,
                               uint32_t* d_count, uint32_t* capped, lcs_stream stream, const uint8_t* only = nullptr);
// lcs_candidates_filter that also drops the pairs whose query vertex (VF: the vertex; EE: the first vertex
// of the query edge) is set in `skip` (optional).
int lcs_candidates_filter_masked(int is_ee, const uint32_t* in_pairs, const uint32_t* in_count, uint32_t in_capacity,
                                 const float* x, const uint32_t* elems, const float* d_hat, const float* thickness,
                                 uint32_t* out_pairs, uint32_t out_capacity, uint32_t* out_count, lcs_stream stream,
                                 const uint8_t* skip);

// DCD pairs straight from the previous iteration's CCD candidate list: the candidates whose static boxes
// overlap at x (the test of lcs_candidates_filter, counted into *d_cand_count) go through the DCD test of
// lcs_dcd_vf / lcs_dcd_ee; the same pairs and counts as filter + DCD without writing the candidate list.
int lcs_dcd_vf_filtered(const uint32_t* ccd_pairs, const uint32_t* d_ccd_count, uint32_t capacity, const float* x,
                        const uint32_t* faces, const uint32_t* body, const float* vert_area, const float* face_area,
                        const float* d_hat, const float* offset, float kappa, lcs_pair* out, uint32_t out_capacity,
                        uint32_t* d_out_count, uint32_t* d_cand_count, lcs_stream stream);
int lcs_dcd_ee_filtered(const uint32_t* ccd_pairs, const uint32_t* d_ccd_count, uint32_t capacity, const float* x,
                        const uint32_t* edges, const uint32_t* body, const float* edge_area, const float* d_hat,
                        const float* offset, float kappa, lcs_pair* out, uint32_t out_capacity, uint32_t* d_out_count,
                        uint32_t* d_cand_count, lcs_stream stream);
