/*
 * lcs_oracle.h -- CPU restatement of the LuisaComputeSimulator contact-and-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is compared
 * against (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm).
 * Nothing in the product links or calls it.
 *
 * Parity status: the reference (LuisaCompute DSL, fetched at configure time) cannot be built
 * here, so this restatement is pinned by the reference's own known answers only:
 *   - Morton32/Morton64 codes of 8 leaves at pos = i/10          (Solver/CollisionDetector/lbvh.cpp:886-897)
 *   - Karras ranges / splits / children / parents of that tree   (Solver/CollisionDetector/lbvh.cpp:561-592)
 *   - complete-tree refit root AABB [0, 2^depth]^3               (UnitTest/test_lbvh_refit.cpp:253-349)
 *   - VF CCD known answer toi = 0.6930697 at offset 1e-3          (Solver/CollisionDetector/narrow_phase.cpp:3282-3307)
 * Everything else is "parity unpinned" against the reference binary and pinned only by this code.
 *
 * Data layout shared with the CUDA path (matches LuisaCompute's Buffer<float3>/Buffer<uint3>):
 *   positions  : float4 per vertex (x, y, z, pad)            16 B
 *   faces      : uint4  per face   (v0, v1, v2, pad)         16 B
 *   edges      : uint2  per edge   (v0, v1)                   8 B
 *   3x3 blocks : 9 floats, column-major (MatrixTriplet3x3 order)
 *   diag 3x3   : 3 float4 columns (Buffer<float3x3> layout)   48 B
 *   contact pair: 48 B CollisionPairTemplate {uint4 idx|type bit31, float4 normal+kappa*area, float4 k1,k2,bary}
 *
 * Floating point: every routine is written so that the order of operations, and every fused
 * multiply-add, is spelled out (fmaf only where written).  Compile with -ffp-contract=off.
 */
#ifndef LCS_ORACLE_H
#define LCS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t idx[4];
    float    vec1[4];
    float    vec2[4];
} orc_pair;

enum { ORC_TREE_VERT = 0, ORC_TREE_EDGE = 1, ORC_TREE_FACE = 2 };

/* ---------------- LBVH (Solver/CollisionDetector/lbvh.cpp) ---------------- */
void orc_morton_codes_unit(uint32_t n, uint32_t* m32, uint64_t* m64);
void orc_lbvh_reduce_aabb(int kind, const float* x, const uint32_t* elems, uint32_t n_elems,
                          uint32_t n_verts, float* gmin3, float* gmax3, float* centers4);
void orc_lbvh_mortons(const float* centers4, uint32_t n, const float* gmin3, const float* gmax3,
                      uint64_t* morton);
void orc_lbvh_sort(const uint64_t* morton, uint32_t n, uint32_t* sorted_get_original,
                   uint64_t* morton_sorted);
int  orc_lbvh_build_inner(const uint64_t* morton_sorted, uint32_t n, uint32_t* parent,
                          uint32_t* children2, int32_t* ranges2, int32_t* splits);
int  orc_lbvh_construct(const uint64_t* morton_sorted, const uint32_t* sorted_get_original,
                        uint32_t n, uint32_t* parent, uint32_t* children2, uint32_t* object_idx);
void orc_lbvh_update_leaves(int kind, const uint32_t* sorted_get_original, uint32_t n,
                            const float* thickness, const float* x0, const float* x1,
                            const uint32_t* elems, float* node_aabb8);
int  orc_lbvh_refit(uint32_t n, const uint32_t* parent, const uint32_t* children2,
                    float* node_aabb8);
uint32_t orc_lbvh_query_vf(uint32_t n_leaves, const float* node_aabb8, const uint32_t* children2,
                           const uint32_t* object_idx, const float* x0, const float* x1,
                           uint32_t n_verts, const float* dhat, const float* thickness,
                           uint32_t* pairs, uint32_t capacity);
uint32_t orc_lbvh_query_ee(uint32_t n_leaves, const float* node_aabb8, const uint32_t* children2,
                           const uint32_t* object_idx, const float* x0, const float* x1,
                           const uint32_t* edges, uint32_t n_edges, const float* dhat,
                           const float* thickness, uint32_t* pairs, uint32_t capacity);

/* ---------------- ACCD / distance (Solver/CollisionDetector/accd.hpp, distance.hpp) -------- */
float orc_point_triangle_ccd(const float* p0, const float* p1, const float* t00, const float* t01,
                             const float* t02, const float* t10, const float* t11,
                             const float* t12, float offset, int fp64_final);
float orc_edge_edge_ccd(const float* ea00, const float* ea01, const float* eb00,
                        const float* eb01, const float* ea10, const float* ea11,
                        const float* eb10, const float* eb11, float offset, int fp64_final);
float orc_pt_dist2(const float* p, const float* t0, const float* t1, const float* t2);
float orc_ee_dist2(const float* a0, const float* a1, const float* b0, const float* b1);
void  orc_pt_coeff(const float* p, const float* t0, const float* t1, const float* t2, float* c3);
void  orc_ee_coeff(const float* a0, const float* a1, const float* b0, const float* b1, float* c4);
void  orc_barrier(float d, float dhat, float* b, float* db, float* ddb);

/* ---------------- narrow phase (Solver/CollisionDetector/narrow_phase.cpp) ---------------- */
float orc_ccd_vf(const uint32_t* pairs, uint32_t n_pairs, const float* x0, const float* x1,
                 const uint32_t* faces, const uint32_t* body, const float* offset,
                 float* toi_per_pair, int fp64_final);
float orc_ccd_ee(const uint32_t* pairs, uint32_t n_pairs, const float* x0, const float* x1,
                 const uint32_t* edges, const uint32_t* body, const float* offset,
                 float* toi_per_pair, int fp64_final);
/* all-FP64 ACCD (every quantity in double; error reference for the precision form, not a
 * restatement of a reference function): is_ee 0 = point (a0) vs triangle (a1..a3) */
double orc_ccd_f64(int is_ee, const float* a0, const float* a1, const float* a2, const float* a3,
                   const float* b0, const float* b1, const float* b2, const float* b3, float offset);
void orc_ccd_f64_list(int is_ee, const uint32_t* pairs, uint32_t n_pairs, const float* x0, const float* x1,
                      const uint32_t* elems, const uint32_t* body, const float* offset, double* toi);
uint32_t orc_dcd_vf(const uint32_t* pairs, uint32_t n_pairs, const float* x, const uint32_t* faces,
                    const uint32_t* body, const float* vert_area, const float* face_area,
                    const float* dhat, const float* offset, float kappa, orc_pair* out,
                    uint32_t capacity);
uint32_t orc_dcd_ee(const uint32_t* pairs, uint32_t n_pairs, const float* x, const uint32_t* edges,
                    const uint32_t* body, const float* edge_area, const float* dhat,
                    const float* offset, float kappa, orc_pair* out, uint32_t capacity);

/* ---------------- contact assembly / energy ---------------- */
void orc_contact_grad_diag(const orc_pair* pairs, uint32_t n, float* b4, float* diag12);
uint32_t orc_contact_offdiag_bsr(const orc_pair* pairs, uint32_t n, uint32_t n_rows,
                                 uint32_t* row_ptr, uint32_t* col, float* val9, uint32_t cap);
double orc_contact_energy(const orc_pair* pairs, uint32_t n, const float* x, const float* dhat,
                          const float* offset, int fp64_sum);

/* ---------------- SpMV + Jacobi PCG (newton_solver.cpp, precond_cg.cpp) ---------------- */
void orc_bsr_spmv(uint32_t n, const float* diag12, const uint32_t* rp_a, const uint32_t* col_a,
                  const float* val_a, const uint32_t* rp_b, const uint32_t* col_b,
                  const float* val_b, const float* x4, float* y4);
typedef struct {
    int32_t iterations;
    float   rel_residual;  /* ||r|| / ||r0|| at exit */
    float   dot_rz;        /* last r.z */
    int32_t status;        /* 0 ok, 1 nan */
} orc_pcg_stats;
int orc_pcg(uint32_t n, const float* diag12, const uint32_t* rp_a, const uint32_t* col_a,
            const float* val_a, const uint32_t* rp_b, const uint32_t* col_b, const float* val_b,
            const float* b4, float* x4, int max_iter, float rel_tol, float abs_rz_tol,
            int check_every, int fp64_dots, orc_pcg_stats* stats);

float orc_min_distance(const uint32_t* vf, uint32_t n_vf, const uint32_t* ee, uint32_t n_ee, const float* x,
                       const uint32_t* faces, const uint32_t* edges);

/* ---------------- material producers of the Newton loop ---------------- */
void orc_material_fill(uint32_t V, uint32_t E, uint32_t B, const float* x4, const float* rest4,
                       const float* xt4, const float* mass, const uint8_t* pinned, float dt,
                       float dirichlet, const uint32_t* edges, const float* rest_len, float spring_k,
                       const float* spring_kper, const uint32_t* stencil, const float* Q16, float bending_k,
                       const uint32_t* spring_slots, const uint32_t* bend_slots, uint32_t nnz,
                       float* b4, float* diag12, float* val9);

/* ---------------- cloth energies (lcs_oracle_material.c) ---------------- */
void orc_bw98_face(const float* x0, const float* x1, const float* x2, const float* dm, float mu, float lambda,
                   float area, float* g9, float* K54);
float orc_dihedral(const float* p0, const float* p1, const float* p2, const float* p3, float* g12);
void orc_eval_stretch_faces(uint32_t n, const float* x4, const uint32_t* faces4, const float* dm4, const float* area,
                            const float* mu_lambda2, float* grad4, float* hess12);
void orc_eval_bending(uint32_t n, const float* x4, const uint32_t* st4, const float* rest_angle, const float* hbar,
                      const float* stiffness, float scaling, float* grad4, float* hess12);
void orc_eval_springs(uint32_t n, const float* x4, const uint32_t* edges2, const float* rest_len,
                      const float* stiffness, float* grad4, float* hess12);
void orc_material_energy(uint32_t V, const float* x4, const float* xt4, const float* mass, const uint8_t* fixed,
                         float dt, float dirichlet, uint32_t E, const uint32_t* springs2, const float* rest_len,
                         const float* spring_k, uint32_t Fs, const uint32_t* faces4, const float* dm4,
                         const float* area, const float* mu_lambda2, uint32_t B, const uint32_t* st4,
                         const float* rest_angle, const float* hbar, const float* bend_k, float scaling, double* out);
void orc_material_fill2(uint32_t V, const float* x4, const float* rest4, const float* xt4, const float* mass,
                        const uint8_t* pinned, float dt, float dirichlet, int stretch_model, int bending_model,
                        uint32_t E, const uint32_t* edges, const float* rest_len, float spring_k, uint32_t Fs,
                        const uint32_t* sfaces4, const float* dm4, const float* sarea, float mu, float lambda,
                        uint32_t B, const uint32_t* stencil, const float* Q16, const float* rest_angle,
                        const float* hbar, float bending_k, float bending_scaling, const uint32_t* spring_slots,
                        const uint32_t* face_slots, const uint32_t* bend_slots, uint32_t nnz, float* b4,
                        float* diag12, float* val9, const float* ml2, const float* bend_kper,
                        const float* spring_kper);

/* ---------------- affine bodies ---------------- */
void orc_contact_grad_diag_abd(const orc_pair* pairs, uint32_t n, const uint32_t* body, const float* model_x4,
                               const uint32_t* body_dof, float* b4, float* diag12);
uint32_t orc_contact_offdiag_bsr_abd(const orc_pair* pairs, uint32_t n, uint32_t n_rows, const uint32_t* body,
                                     const float* model_x4, const uint32_t* body_dof, uint32_t* row_ptr, uint32_t* col,
                                     float* val9, uint32_t cap);
void orc_abd_fill(uint32_t NB, const uint32_t* body_dof, const float* mass16, const float* volume, const float* kappa,
                  const uint8_t* fixed, const float* x4, const float* xt4, float dt, float dirichlet,
                  const uint32_t* body_slots, float* b4, float* diag12, float* val9);

#ifdef __cplusplus
}
#endif
#endif
