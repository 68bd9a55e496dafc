"""ctypes binding of liblcs_b200.so (the C ABI declared in include/lcs_gpu.h).

Loading the library needs no GPU; calling its compute entry points does.  There is no CPU
fallback: if the library is missing the import of this module fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblcs_b200.so")

P = C.c_void_p
U32 = C.c_uint32
I32 = C.c_int
F32 = C.c_float


class LcsError(RuntimeError):
    pass


STATUS = {0: "LCS_OK", 1: "LCS_ERR_INVALID", 2: "LCS_ERR_CUDA", 3: "LCS_ERR_CAPACITY", 4: "LCS_ERR_UNHEALTHY_BVH",
          5: "LCS_ERR_NAN", 6: "LCS_ERR_CCD_NOCONVERGE", 7: "LCS_ERR_TIMEOUT", 8: "LCS_ERR_NO_DEVICE",
          9: "LCS_ERR_LINESEARCH"}
LCS_TREE_VERT, LCS_TREE_EDGE, LCS_TREE_FACE = 0, 1, 2
LCS_CCD_FP64_FINAL, LCS_CCD_FP64 = 1, 2
LCS_PCG_FP64_DOTS, LCS_PCG_PLAIN, LCS_PCG_NO_STATS, LCS_PCG_ROWS, LCS_PCG_SINGLE_REDUCTION = 1, 2, 4, 8, 16
LCS_STRETCH_SPRING, LCS_STRETCH_BW98 = 0, 1
LCS_BENDING_NONE, LCS_BENDING_QUADRATIC, LCS_BENDING_DIHEDRAL = 0, 1, 2


class Bsr(C.Structure):
    _fields_ = [("n_rows", C.c_uint32), ("row_ptr", P), ("col", P), ("val", P)]


class PcgOpts(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("rel_tol", C.c_float), ("abs_rz_tol", C.c_float),
                ("check_every", C.c_int32), ("flags", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("n_verts", C.c_uint32), ("n_faces", C.c_uint32), ("n_edges", C.c_uint32), ("n_bending", C.c_uint32),
                ("x", P), ("v", P), ("faces", P), ("edges", P), ("bending", P), ("bending_Q", P), ("rest_len", P),
                ("vert_area", P), ("face_area", P), ("edge_area", P), ("mass", P), ("d_hat", P), ("offset", P),
                ("body", P), ("pinned", P), ("anim_group", P), ("n_anim", C.c_uint32), ("anim", P),
                ("dt", C.c_float), ("gravity", C.c_float * 3), ("kappa", C.c_float), ("spring_k", C.c_float),
                ("bending_k", C.c_float), ("dirichlet", C.c_float), ("damping", C.c_float),
                ("use_floor", C.c_int32), ("floor_y", C.c_float), ("nonlinear_iters", C.c_int32),
                ("pcg_max_iter", C.c_int32), ("pcg_rel_tol", C.c_float), ("pcg_abs_rz_tol", C.c_float),
                ("pcg_check_every", C.c_int32), ("stretch_model", C.c_int32), ("bending_model", C.c_int32),
                ("n_stretch_faces", C.c_uint32), ("stretch_faces", P), ("stretch_dm_inv", P), ("stretch_area", P),
                ("stretch_mu", C.c_float), ("stretch_lambda", C.c_float), ("bending_rest_angle", P),
                ("bending_hbar", P), ("bending_scaling", C.c_float), ("n_bodies", C.c_uint32), ("body_dof", P),
                ("body_mass", P), ("body_volume", P), ("body_kappa", P), ("model_x", P),
                ("stretch_mu_lambda", P), ("bending_stiffness", P), ("spring_stiffness", P)]


class AbdView(C.Structure):
    _fields_ = [("body", P), ("model_x", P), ("body_dof", P)]


class ClothElements(C.Structure):
    _fields_ = [("n_verts", C.c_uint32), ("n_springs", C.c_uint32), ("n_stretch_faces", C.c_uint32),
                ("n_bending", C.c_uint32), ("mass", P), ("is_fixed", P), ("springs", P), ("spring_rest_len", P),
                ("spring_stiffness", P), ("stretch_faces", P), ("stretch_dm_inv", P), ("stretch_area", P),
                ("stretch_mu_lambda", P), ("bending_edges", P), ("bending_rest_angle", P), ("bending_hbar", P),
                ("bending_stiffness", P), ("bending_scaling", C.c_float)]


class NewtonStats(C.Structure):
    _fields_ = [("newton_iters", C.c_int32), ("pcg_iters", C.c_int32), ("last_toi", C.c_float),
                ("last_rel_residual", C.c_float), ("vf_candidates", C.c_uint32), ("ee_candidates", C.c_uint32),
                ("contact_pairs", C.c_uint32), ("ccd_vf_candidates", C.c_uint32),
                ("ccd_ee_candidates", C.c_uint32), ("status", C.c_int32), ("retries", C.c_int32),
                ("host_ms", C.c_float), ("last_alpha", C.c_float), ("ls_halvings", C.c_int32)]


class BvhDataView(C.Structure):
    _fields_ = [("n_leaves", C.c_uint32), ("parent", P), ("children", P), ("morton_sorted", P),
                ("sorted_get_original", P), ("is_healthy", P)]


class IterRecord(C.Structure):
    _fields_ = [("pcg_iters", C.c_int32), ("rel_residual", C.c_float), ("toi", C.c_float), ("max_dx", C.c_float),
                ("vf_candidates", C.c_uint32), ("ee_candidates", C.c_uint32), ("contact_pairs", C.c_uint32),
                ("ccd_vf_candidates", C.c_uint32), ("ccd_ee_candidates", C.c_uint32)]


class PcgStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("rel_residual", C.c_float), ("dot_rz", C.c_float),
                ("status", C.c_int32)]


# name -> (restype, argtypes); must list every function of include/lcs_gpu.h
SIGNATURES = {
    "lcs_version": (C.c_char_p, []),
    "lcs_device_check": (I32, [I32]),
    "lcs_last_error": (C.c_char_p, []),
    "lcs_launch_count": (C.c_uint64, []),
    "lcs_bvh_create": (I32, [I32, U32, C.POINTER(P)]),
    "lcs_bvh_destroy": (I32, [P]),
    "lcs_debug_pcg_wait": (I32, [I32, I32, U32, U32, P]),
    "lcs_forest_query_tuning": (I32, [P, P, P]),
    "lcs_newton_batch_query_tuning": (I32, [P, P, P]),
    "lcs_bvh_check_construction": (I32, [P, P]),
    "lcs_bvh_data": (I32, [P, P]),
    "lcs_bvh_reduce_aabb": (I32, [P, P, P, U32, P]),
    "lcs_bvh_construct": (I32, [P, P]),
    "lcs_bvh_update_leaves": (I32, [P, P, P, P, P, P]),
    "lcs_bvh_refit": (I32, [P, P]),
    "lcs_bvh_update_refit": (I32, [P, P, P, P, P, P]),
    "lcs_bvh_query_vf": (I32, [P, P, P, U32, P, P, P, U32, P, P]),
    "lcs_bvh_query_ee": (I32, [P, P, P, P, U32, P, P, P, U32, P, P]),
    "lcs_bvh_query_ee_sym": (I32, [P, P, P, P, C.c_float, P, U32, P, P]),
    "lcs_bvh_health": (I32, [P, C.POINTER(C.c_int), P]),
    "lcs_bvh_export": (I32, [P, P, P, P, P, P, P, P, P, P]),
    "lcs_bvh_num_leaves": (U32, [P]),
    "lcs_ccd_vf": (I32, [P, P, U32, P, P, P, P, P, P, P, I32, P]),
    "lcs_ccd_ee": (I32, [P, P, U32, P, P, P, P, P, P, P, I32, P]),
    "lcs_dcd_vf": (I32, [P, P, U32, P, P, P, P, P, P, P, F32, P, U32, P, P]),
    "lcs_dcd_ee": (I32, [P, P, U32, P, P, P, P, P, P, F32, P, U32, P, P]),
    "lcs_contact_grad_diag": (I32, [P, P, U32, P, P, P]),
    "lcs_contact_grad_diag_abd": (I32, [P, P, U32, P, P, C.POINTER(AbdView), P]),
    "lcs_assembler_create_abd": (I32, [U32, U32, C.POINTER(P)]),
    "lcs_contact_offdiag_bsr_abd": (I32, [P, P, P, U32, C.POINTER(AbdView), P]),
    "lcs_contact_energy": (I32, [P, P, U32, P, P, P, P, P]),
    "lcs_assembler_create": (I32, [U32, U32, C.POINTER(P)]),
    "lcs_assembler_destroy": (I32, [P]),
    "lcs_contact_offdiag_bsr": (I32, [P, P, P, U32, P]),
    "lcs_assembler_bsr": (I32, [P, C.POINTER(Bsr), C.POINTER(P)]),
    "lcs_assembler_export": (I32, [P, P, P, P, U32, C.POINTER(C.c_uint32), P]),
    "lcs_spmv": (I32, [U32, P, C.POINTER(Bsr), C.POINTER(Bsr), P, P, P]),
    "lcs_pcg_create": (I32, [U32, C.POINTER(P)]),
    "lcs_pcg_destroy": (I32, [P]),
    "lcs_pcg_solve": (I32, [P, P, C.POINTER(Bsr), C.POINTER(Bsr), P, P, C.POINTER(PcgOpts), C.POINTER(PcgStats), P]),
    "lcs_pcg_device_stats": (P, [P]),
    "lcs_pcg_solve_noalloc": (I32, [U32, P, C.POINTER(Bsr), C.POINTER(Bsr), P, P, C.POINTER(PcgOpts),
                                    C.POINTER(PcgStats), P]),
    "lcs_eval_springs": (I32, [P, P, P, P, U32, P, P, P]),
    "lcs_eval_stretch_faces": (I32, [P, P, P, P, P, U32, P, P, P]),
    "lcs_eval_bending": (I32, [P, P, P, P, P, F32, U32, P, P, P]),
    "lcs_material_energy": (I32, [C.POINTER(ClothElements), P, P, F32, F32, P, P]),
    "lcs_newton_create": (I32, [C.POINTER(SceneDesc), I32, P, C.POINTER(P)]),
    "lcs_newton_create_batch": (I32, [C.POINTER(SceneDesc), U32, I32, P, I32, C.POINTER(P)]),
    "lcs_newton_num_scenes": (U32, [P]),
    "lcs_newton_scene_stats": (I32, [P, U32, C.POINTER(NewtonStats)]),
    "lcs_newton_download_scene": (I32, [P, U32, P, P]),
    "lcs_forest_create": (I32, [I32, U32, P, P, C.POINTER(P)]),
    "lcs_forest_destroy": (I32, [P]),
    "lcs_forest_build": (I32, [P, P, P, P]),
    "lcs_forest_update_refit": (I32, [P, P, P, P, P, P]),
    "lcs_forest_query_vf": (I32, [P, P, P, U32, P, P, P, P, U32, P, P]),
    "lcs_forest_query_ee": (I32, [P, P, P, P, P, P, P, U32, P, P]),
    "lcs_forest_health": (I32, [P, C.POINTER(C.c_int), P]),
    "lcs_forest_export_scene": (I32, [P, U32, P, P, P, P, P, P, P, P]),
    "lcs_candidates_filter": (I32, [I32, P, P, U32, P, P, P, P, P, U32, P, P]),
    "lcs_ccd_batch": (I32, [I32, P, P, U32, P, P, P, P, P, P, P, P, I32, P]),
    "lcs_pcg_solve_batch": (I32, [P, U32, P, P, P, P, C.POINTER(Bsr), C.POINTER(Bsr), P, P,
                                  C.POINTER(PcgOpts), P, I32, P]),
    "lcs_pcg_batch_tuning": (I32, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_float)]),
    "lcs_newton_destroy": (I32, [P]),
    "lcs_newton_last_iterate": (I32, [P, P, P, P]),
    "lcs_newton_step": (I32, [P, C.POINTER(NewtonStats)]),
    "lcs_newton_step_host": (I32, [P, P, P, P, P, C.POINTER(NewtonStats)]),
    "lcs_newton_state": (I32, [P, C.POINTER(P), C.POINTER(P)]),
    "lcs_newton_download": (I32, [P, P, P]),
    "lcs_newton_upload": (I32, [P, P, P]),
    "lcs_newton_invalidate": (I32, [P]),
    "lcs_newton_set_frame": (I32, [P, U32]),
    "lcs_newton_iteration_log": (I32, [P, P, I32, P]),
    "lcs_newton_get_frame": (I32, [P, P]),
    "lcs_newton_profile": (I32, [P, C.POINTER(C.c_double), C.POINTER(C.c_int32), I32]),
    "lcs_newton_reset_profile": (I32, [P]),
    "lcs_newton_pcg_kind": (I32, [P]),
    "lcs_newton_batch_tuning": (I32, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_float)]),
    "lcs_newton_counts": (I32, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                C.POINTER(C.c_uint32)]),
}
LCS_NEWTON_PLAIN, LCS_NEWTON_FP64, LCS_NEWTON_PROFILE, LCS_NEWTON_PCG_SINGLE_REDUCTION, LCS_NEWTON_FULL_TRAVERSAL = \
    1, 2, 4, 8, 16
LCS_NEWTON_ENERGY_LINESEARCH = 32
LCS_NEWTON_PCG_GLOBAL_MATRIX = 64
LCS_NEWTON_DETERMINISTIC = 128
PHASES = ["build", "material", "dcd_broad", "dcd_narrow", "assembly", "pcg", "ccd_broad", "ccd_narrow", "apply"]

_lib = None


def load():
    """Loads liblcs_b200.so (building it first when the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(code, what=""):
    if code != 0:
        msg = load().lcs_last_error().decode(errors="replace")
        raise LcsError(f"{what}: {STATUS.get(code, code)} {msg}")
    return code
