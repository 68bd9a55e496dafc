"""ctypes wrapper of the CPU oracle (oracle/lcs_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference arm, never by the product package.  The oracle is the checker the
CUDA path is compared with; see lcs_oracle.h for the layouts and which reference known
answers pin it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liblcs_oracle.so")
_lib = None

PAIR_DTYPE = np.dtype([("idx", "<u4", (4,)), ("vec1", "<f4", (4,)), ("vec2", "<f4", (4,))])
TREE_VERT, TREE_EDGE, TREE_FACE = 0, 1, 2


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < max(
        os.path.getmtime(os.path.join(_HERE, f))
        for f in ("lcs_oracle.c", "lcs_oracle.h", "lcs_oracle_geom.inc", "Makefile")
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_SO)
        _declare(_lib)
    return _lib


P = C.c_void_p
U32 = C.c_uint32
F32 = C.c_float
I32 = C.c_int


class PcgStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("rel_residual", C.c_float),
                ("dot_rz", C.c_float), ("status", C.c_int32)]


def _declare(L):
    sig = {
        "orc_morton_codes_unit": (None, [U32, P, P]),
        "orc_lbvh_reduce_aabb": (None, [I32, P, P, U32, U32, P, P, P]),
        "orc_lbvh_mortons": (None, [P, U32, P, P, P]),
        "orc_lbvh_sort": (None, [P, U32, P, P]),
        "orc_lbvh_build_inner": (I32, [P, U32, P, P, P, P]),
        "orc_lbvh_construct": (I32, [P, P, U32, P, P, P]),
        "orc_lbvh_update_leaves": (None, [I32, P, U32, P, P, P, P, P]),
        "orc_lbvh_refit": (I32, [U32, P, P, P]),
        "orc_lbvh_query_vf": (U32, [U32, P, P, P, P, P, U32, P, P, P, U32]),
        "orc_lbvh_query_ee": (U32, [U32, P, P, P, P, P, P, U32, P, P, P, U32]),
        "orc_point_triangle_ccd": (F32, [P, P, P, P, P, P, P, P, F32, I32]),
        "orc_edge_edge_ccd": (F32, [P, P, P, P, P, P, P, P, F32, I32]),
        "orc_pt_dist2": (F32, [P, P, P, P]),
        "orc_ee_dist2": (F32, [P, P, P, P]),
        "orc_pt_coeff": (None, [P, P, P, P, P]),
        "orc_ee_coeff": (None, [P, P, P, P, P]),
        "orc_barrier": (None, [F32, F32, P, P, P]),
        "orc_ccd_vf": (F32, [P, U32, P, P, P, P, P, P, I32]),
        "orc_ccd_ee": (F32, [P, U32, P, P, P, P, P, P, I32]),
        "orc_ccd_f64_list": (None, [I32, P, U32, P, P, P, P, P, P]),
        "orc_dcd_vf": (U32, [P, U32, P, P, P, P, P, P, P, F32, P, U32]),
        "orc_dcd_ee": (U32, [P, U32, P, P, P, P, P, P, F32, P, U32]),
        "orc_contact_grad_diag": (None, [P, U32, P, P]),
        "orc_contact_offdiag_bsr": (U32, [P, U32, U32, P, P, P, U32]),
        "orc_contact_energy": (C.c_double, [P, U32, P, P, P, I32]),
        "orc_bsr_spmv": (None, [U32, P, P, P, P, P, P, P, P, P]),
        "orc_material_fill": (None, [U32, U32, U32, P, P, P, P, P, F32, F32, P, P, F32, P, P, P, F32, P, P, U32, P,
                                     P, P]),
        "orc_min_distance": (F32, [P, U32, P, U32, P, P, P]),
        "orc_bw98_face": (None, [P, P, P, P, F32, F32, F32, P, P]),
        "orc_dihedral": (F32, [P, P, P, P, P]),
        "orc_eval_stretch_faces": (None, [U32, P, P, P, P, P, P, P]),
        "orc_eval_bending": (None, [U32, P, P, P, P, P, F32, P, P]),
        "orc_eval_springs": (None, [U32, P, P, P, P, P, P]),
        "orc_material_energy": (None, [U32, P, P, P, P, F32, F32, U32, P, P, P, U32, P, P, P, P, U32, P, P, P, P, F32,
                                       P]),
        "orc_contact_grad_diag_abd": (None, [P, U32, P, P, P, P, P]),
        "orc_contact_offdiag_bsr_abd": (U32, [P, U32, U32, P, P, P, P, P, P, U32]),
        "orc_abd_fill": (None, [U32, P, P, P, P, P, P, P, F32, F32, P, P, P, P]),
        "orc_material_fill2": (None, [U32, P, P, P, P, P, F32, F32, I32, I32, U32, P, P, F32, U32, P, P, P, F32, F32,
                                      U32, P, P, P, P, F32, F32, P, P, P, U32, P, P, P, P, P, P]),
        "orc_pcg": (I32, [U32, P, P, P, P, P, P, P, P, P, I32, F32, F32, I32, I32, C.POINTER(PcgStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def f4(x):
    """(n,3) or (n,4) float array -> (n,4) float32 contiguous (pad = 0)."""
    x = np.asarray(x, dtype=np.float32)
    if x.shape[1] == 4:
        return np.ascontiguousarray(x)
    out = np.zeros((x.shape[0], 4), np.float32)
    out[:, :3] = x
    return out


def u4(faces):
    faces = np.asarray(faces, dtype=np.uint32)
    if faces.shape[1] == 4:
        return np.ascontiguousarray(faces)
    out = np.zeros((faces.shape[0], 4), np.uint32)
    out[:, :3] = faces
    return out


# ----------------------------------------------------------------------------------- LBVH
def morton_unit(n=8):
    m32 = np.zeros(n, np.uint32)
    m64 = np.zeros(n, np.uint64)
    lib().orc_morton_codes_unit(n, _p(m32), _p(m64))
    return m32, m64


def build_inner(morton_sorted):
    ms = np.ascontiguousarray(morton_sorted, dtype=np.uint64)
    n = ms.shape[0]
    parent = np.full(2 * n - 1, 0xFFFFFFFF, np.uint32)
    children = np.zeros((2 * n - 1, 2), np.uint32)
    ranges = np.zeros((max(n - 1, 1), 2), np.int32)
    splits = np.zeros(max(n - 1, 1), np.int32)
    ok = lib().orc_lbvh_build_inner(_p(ms), n, _p(parent), _p(children), _p(ranges), _p(splits))
    return dict(parent=parent, children=children, ranges=ranges[: n - 1], splits=splits[: n - 1], healthy=ok)


class Tree:
    """Everything the reference's LbvhData holds for one tree (lbvh.h:79-152)."""

    def __init__(self, kind, n_leaves):
        self.kind, self.n = kind, n_leaves


def lbvh_build(kind, x, elems, n_verts):
    """reduce_*_tree_aabb + construct_tree: returns a Tree with topology (lbvh.cpp:939-998)."""
    x = f4(x)
    elems = np.ascontiguousarray(elems, np.uint32) if elems is not None else None
    n = n_verts if kind == TREE_VERT else elems.shape[0]
    L = lib()
    gmin = np.zeros(3, np.float32)
    gmax = np.zeros(3, np.float32)
    centers = np.zeros((n, 4), np.float32)
    L.orc_lbvh_reduce_aabb(kind, _p(x), _p(elems), n, n_verts, _p(gmin), _p(gmax), _p(centers))
    morton = np.zeros(n, np.uint64)
    L.orc_lbvh_mortons(_p(centers), n, _p(gmin), _p(gmax), _p(morton))
    sgo = np.zeros(n, np.uint32)
    ms = np.zeros(n, np.uint64)
    L.orc_lbvh_sort(_p(morton), n, _p(sgo), _p(ms))
    nn = max(2 * n - 1, 1)
    parent = np.full(nn, 0xFFFFFFFF, np.uint32)
    children = np.zeros((nn, 2), np.uint32)
    obj = np.full(nn, 0xFFFFFFFF, np.uint32)
    ok = L.orc_lbvh_construct(_p(ms), _p(sgo), n, _p(parent), _p(children), _p(obj))
    t = Tree(kind, n)
    t.gmin, t.gmax, t.morton, t.morton_sorted, t.sorted_get_original = gmin, gmax, morton, ms, sgo
    t.parent, t.children, t.object_idx, t.healthy = parent, children, obj, ok
    t.node_aabb = np.zeros((nn, 8), np.float32)
    t.elems = elems
    return t


def lbvh_refit(t, x0, x1, elems, thickness):
    """update_*_tree_leave_aabb + refit (lbvh.cpp:1001-1045)."""
    L = lib()
    x0, x1 = f4(x0), f4(x1)
    thickness = np.ascontiguousarray(thickness, np.float32)
    e = np.ascontiguousarray(elems, np.uint32) if elems is not None else None
    L.orc_lbvh_update_leaves(t.kind, _p(t.sorted_get_original), t.n, _p(thickness), _p(x0), _p(x1),
                             _p(e), _p(t.node_aabb))
    return L.orc_lbvh_refit(t.n, _p(t.parent), _p(t.children), _p(t.node_aabb))


def lbvh_query_vf(t, x0, x1, dhat, thickness, capacity=None):
    x0, x1 = f4(x0), f4(x1)
    nv = x0.shape[0]
    cap = capacity if capacity is not None else 64 * nv + 1024
    pairs = np.zeros((cap, 2), np.uint32)
    cnt = lib().orc_lbvh_query_vf(t.n, _p(t.node_aabb), _p(t.children), _p(t.object_idx), _p(x0), _p(x1),
                                  nv, _p(np.ascontiguousarray(dhat, np.float32)),
                                  _p(np.ascontiguousarray(thickness, np.float32)), _p(pairs), cap)
    if capacity is None and cnt > cap:
        return lbvh_query_vf(t, x0, x1, dhat, thickness, capacity=int(cnt))
    return pairs[: min(cnt, cap)], int(cnt)


def lbvh_query_ee(t, x0, x1, edges, dhat, thickness, capacity=None):
    x0, x1 = f4(x0), f4(x1)
    edges = np.ascontiguousarray(edges, np.uint32)
    ne = edges.shape[0]
    cap = capacity if capacity is not None else 64 * ne + 1024
    pairs = np.zeros((cap, 2), np.uint32)
    cnt = lib().orc_lbvh_query_ee(t.n, _p(t.node_aabb), _p(t.children), _p(t.object_idx), _p(x0), _p(x1),
                                  _p(edges), ne, _p(np.ascontiguousarray(dhat, np.float32)),
                                  _p(np.ascontiguousarray(thickness, np.float32)), _p(pairs), cap)
    if capacity is None and cnt > cap:
        return lbvh_query_ee(t, x0, x1, edges, dhat, thickness, capacity=int(cnt))
    return pairs[: min(cnt, cap)], int(cnt)


# ----------------------------------------------------------------------------- ACCD / DCD
def _v(a):
    return np.ascontiguousarray(a, np.float32)


def point_triangle_ccd(p0, p1, t00, t01, t02, t10, t11, t12, offset, fp64_final=False):
    a = [_v(v) for v in (p0, p1, t00, t01, t02, t10, t11, t12)]
    return lib().orc_point_triangle_ccd(*[_p(v) for v in a], float(offset), int(fp64_final))


def edge_edge_ccd(ea00, ea01, eb00, eb01, ea10, ea11, eb10, eb11, offset, fp64_final=False):
    a = [_v(v) for v in (ea00, ea01, eb00, eb01, ea10, ea11, eb10, eb11)]
    return lib().orc_edge_edge_ccd(*[_p(v) for v in a], float(offset), int(fp64_final))


def barrier(d, dhat):
    b, db, ddb = C.c_float(), C.c_float(), C.c_float()
    lib().orc_barrier(float(d), float(dhat), C.byref(b), C.byref(db), C.byref(ddb))
    return b.value, db.value, ddb.value


def ccd_vf(pairs, x0, x1, faces, body, offset, per_pair=True, fp64_final=False):
    pairs = np.ascontiguousarray(pairs, np.uint32)
    n = pairs.shape[0]
    toi = np.zeros(n, np.float32) if per_pair else None
    g = lib().orc_ccd_vf(_p(pairs), n, _p(f4(x0)), _p(f4(x1)), _p(u4(faces)),
                         _p(np.ascontiguousarray(body, np.uint32)), _p(_v(offset)), _p(toi), int(fp64_final))
    return g, toi


def ccd_ee(pairs, x0, x1, edges, body, offset, per_pair=True, fp64_final=False):
    pairs = np.ascontiguousarray(pairs, np.uint32)
    n = pairs.shape[0]
    toi = np.zeros(n, np.float32) if per_pair else None
    g = lib().orc_ccd_ee(_p(pairs), n, _p(f4(x0)), _p(f4(x1)), _p(np.ascontiguousarray(edges, np.uint32)),
                         _p(np.ascontiguousarray(body, np.uint32)), _p(_v(offset)), _p(toi), int(fp64_final))
    return g, toi


def ccd_f64(is_ee, pairs, x0, x1, elems, body, offset):
    """Per-pair TOI of the same ACCD iteration carried out entirely in double precision (the
    error reference of the precision form).  elems: faces (n, 4) for VF, edges (n, 2) for EE."""
    pairs = np.ascontiguousarray(pairs, np.uint32)
    n = pairs.shape[0]
    toi = np.zeros(max(n, 1), np.float64)
    el = u4(elems) if not is_ee else np.ascontiguousarray(elems, np.uint32)
    lib().orc_ccd_f64_list(int(is_ee), _p(pairs), n, _p(f4(x0)), _p(f4(x1)), _p(el),
                           _p(np.ascontiguousarray(body, np.uint32)), _p(_v(offset)), _p(toi))
    return toi[:n]


def dcd_vf(pairs, x, faces, body, vert_area, face_area, dhat, offset, kappa):
    pairs = np.ascontiguousarray(pairs, np.uint32)
    n = pairs.shape[0]
    out = np.zeros(max(n, 1), PAIR_DTYPE)
    cnt = lib().orc_dcd_vf(_p(pairs), n, _p(f4(x)), _p(u4(faces)), _p(np.ascontiguousarray(body, np.uint32)),
                           _p(_v(vert_area)), _p(_v(face_area)), _p(_v(dhat)), _p(_v(offset)), float(kappa),
                           _p(out), out.shape[0])
    return out[:cnt]


def dcd_ee(pairs, x, edges, body, edge_area, dhat, offset, kappa):
    pairs = np.ascontiguousarray(pairs, np.uint32)
    n = pairs.shape[0]
    out = np.zeros(max(n, 1), PAIR_DTYPE)
    cnt = lib().orc_dcd_ee(_p(pairs), n, _p(f4(x)), _p(np.ascontiguousarray(edges, np.uint32)),
                           _p(np.ascontiguousarray(body, np.uint32)), _p(_v(edge_area)), _p(_v(dhat)),
                           _p(_v(offset)), float(kappa), _p(out), out.shape[0])
    return out[:cnt]


# --------------------------------------------------------------------- assembly / PCG
def contact_grad_diag(pairs, n_verts, b=None, diag=None):
    pairs = np.ascontiguousarray(pairs, PAIR_DTYPE)
    b = np.zeros((n_verts, 4), np.float32) if b is None else np.ascontiguousarray(b, np.float32).copy()
    diag = np.zeros((n_verts, 3, 4), np.float32) if diag is None else np.ascontiguousarray(diag, np.float32).copy()
    lib().orc_contact_grad_diag(_p(pairs), pairs.shape[0], _p(b), _p(diag))
    return b, diag


def contact_offdiag_bsr(pairs, n_rows):
    pairs = np.ascontiguousarray(pairs, PAIR_DTYPE)
    cap = 12 * max(pairs.shape[0], 1)
    rp = np.zeros(n_rows + 1, np.uint32)
    col = np.zeros(cap, np.uint32)
    val = np.zeros((cap, 9), np.float32)
    nb = lib().orc_contact_offdiag_bsr(_p(pairs), pairs.shape[0], n_rows, _p(rp), _p(col), _p(val), cap)
    return rp, col[:nb], val[:nb]


def _abd_args(sc):
    return (np.ascontiguousarray(sc.body, np.uint32), f4(sc.model_x), np.ascontiguousarray(sc.body_dof, np.uint32))


def contact_grad_diag_abd(pairs, sc, b, diag):
    """contact_grad_diag with the affine-body remap (a rigid side adds to its body's DOF slots)."""
    pairs = np.ascontiguousarray(pairs, PAIR_DTYPE)
    b = np.ascontiguousarray(b, np.float32).copy()
    diag = np.ascontiguousarray(diag, np.float32).copy()
    body, mx, dof = _abd_args(sc)
    lib().orc_contact_grad_diag_abd(_p(pairs), pairs.shape[0], _p(body), _p(mx), _p(dof), _p(b), _p(diag))
    return b, diag


def contact_offdiag_bsr_abd(pairs, sc):
    pairs = np.ascontiguousarray(pairs, PAIR_DTYPE)
    n_rows = sc.num_verts
    cap = 56 * max(pairs.shape[0], 1)
    rp = np.zeros(n_rows + 1, np.uint32)
    col = np.zeros(cap, np.uint32)
    val = np.zeros((cap, 9), np.float32)
    body, mx, dof = _abd_args(sc)
    nb = lib().orc_contact_offdiag_bsr_abd(_p(pairs), pairs.shape[0], n_rows, _p(body), _p(mx), _p(dof), _p(rp),
                                           _p(col), _p(val), cap)
    return rp, col[:nb], val[:nb]


def contact_energy(pairs, x, dhat, offset, fp64=True):
    pairs = np.ascontiguousarray(pairs, PAIR_DTYPE)
    return lib().orc_contact_energy(_p(pairs), pairs.shape[0], _p(f4(x)), _p(_v(dhat)), _p(_v(offset)), int(fp64))


def _bsr_args(m):
    if m is None:
        return None, None, None
    rp, col, val = m
    return (np.ascontiguousarray(rp, np.uint32), np.ascontiguousarray(col, np.uint32),
            np.ascontiguousarray(val, np.float32))


def bsr_spmv(diag, A, B, x):
    x = f4(x)
    n = x.shape[0]
    y = np.zeros((n, 4), np.float32)
    a, b = _bsr_args(A), _bsr_args(B)
    lib().orc_bsr_spmv(n, _p(np.ascontiguousarray(diag, np.float32)), *[_p(v) for v in a], *[_p(v) for v in b],
                       _p(x), _p(y))
    return y


def pcg(diag, A, B, b, max_iter=100, rel_tol=1e-4, abs_rz_tol=1e-10, check_every=25, fp64_dots=False):
    b = f4(b)
    n = b.shape[0]
    x = np.zeros((n, 4), np.float32)
    a_, b_ = _bsr_args(A), _bsr_args(B)
    st = PcgStats()
    lib().orc_pcg(n, _p(np.ascontiguousarray(diag, np.float32)), *[_p(v) for v in a_], *[_p(v) for v in b_],
                  _p(b), _p(x), int(max_iter), float(rel_tol), float(abs_rz_tol), int(check_every),
                  int(fp64_dots), C.byref(st))
    return x, dict(iterations=st.iterations, rel_residual=st.rel_residual, dot_rz=st.dot_rz, status=st.status)


def min_distance(sc, x, radius=5e-3):
    """Smallest VF / EE distance of the mesh at x (candidates within `radius`); > 0 means no
    intersection (device_post_dist_check, newton_solver.cpp:3364-3375)."""
    x = f4(x)
    r = np.full(sc.num_verts, radius, np.float32)
    r[np.asarray(sc.d_hat) < 0] = -1.0  # affine-body DOF slots query nothing
    z = np.zeros(sc.num_verts, np.float32)
    tf = lbvh_build(TREE_FACE, x, sc.faces, sc.num_verts)
    lbvh_refit(tf, x, x, sc.faces, z)
    vf, _ = lbvh_query_vf(tf, x, x, r, z)
    te = lbvh_build(TREE_EDGE, x, sc.edges, sc.num_verts)
    lbvh_refit(te, x, x, sc.edges, z)
    ee, _ = lbvh_query_ee(te, x, x, sc.edges, r, z)
    vf = np.ascontiguousarray(vf, np.uint32)
    ee = np.ascontiguousarray(ee, np.uint32)
    return lib().orc_min_distance(_p(vf), vf.shape[0], _p(ee), ee.shape[0], _p(x), _p(u4(sc.faces)),
                                  _p(np.ascontiguousarray(sc.edges, np.uint32)))


# --------------------------------------------------------------------------- cloth energies
def eval_stretch_faces(x, faces4, dm4, area, mu_lambda):
    """orc_eval_stretch_faces: per face 3 gradients (float4) and 9 Hessian blocks (3 float4 columns)."""
    n = faces4.shape[0]
    g = np.zeros((n, 3, 4), np.float32)
    h = np.zeros((n, 9, 3, 4), np.float32)
    c = np.ascontiguousarray
    lib().orc_eval_stretch_faces(n, _p(f4(x)), _p(u4(faces4)), _p(c(dm4, np.float32)), _p(c(area, np.float32)),
                                 _p(c(mu_lambda, np.float32)), _p(g), _p(h))
    return g, h


def eval_bending(x, stencils, rest_angle, hbar, stiffness, scaling):
    """orc_eval_bending: per stencil 4 gradients and 16 Hessian blocks."""
    n = stencils.shape[0]
    g = np.zeros((n, 4, 4), np.float32)
    h = np.zeros((n, 16, 3, 4), np.float32)
    c = np.ascontiguousarray
    lib().orc_eval_bending(n, _p(f4(x)), _p(c(stencils, np.uint32)), _p(c(rest_angle, np.float32)),
                           _p(c(hbar, np.float32)), _p(c(stiffness, np.float32)), float(scaling), _p(g), _p(h))
    return g, h


def eval_springs(x, edges, rest_len, stiffness):
    n = edges.shape[0]
    g = np.zeros((n, 2, 4), np.float32)
    h = np.zeros((n, 4, 3, 4), np.float32)
    c = np.ascontiguousarray
    lib().orc_eval_springs(n, _p(f4(x)), _p(c(edges, np.uint32)), _p(c(rest_len, np.float32)),
                           _p(c(stiffness, np.float32)), _p(g), _p(h))
    return g, h


def bw98_face(x0, x1, x2, dm, mu, lam, area):
    """orc_bw98_face on one triangle: gradient (3, 3) and blocks (6, 9) [(0,0) (1,1) (2,2) (0,1) (0,2) (1,2)]."""
    f = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    g = np.zeros(9, np.float32)
    K = np.zeros(54, np.float32)
    lib().orc_bw98_face(_p(f(x0)), _p(f(x1)), _p(f(x2)), _p(f(dm)), float(mu), float(lam), float(area), _p(g), _p(K))
    return g.reshape(3, 3), K.reshape(6, 9)


def dihedral(p0, p1, p2, p3):
    f = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    g = np.zeros(12, np.float32)
    th = lib().orc_dihedral(_p(f(p0)), _p(f(p1)), _p(f(p2)), _p(f(p3)), _p(g))
    return th, g.reshape(4, 3)


def material_energy(sc, x, x_tilde, dt):
    """orc_material_energy of a scene: [inertia, springs, stretch faces, bending] in double."""
    c = np.ascontiguousarray
    out = np.zeros(4, np.float64)
    spring = sc.stretch_model == 0
    bw = sc.stretch_model == 1
    dih = sc.bending_model == 2
    E = sc.edges.shape[0] if spring else 0
    Fs = sc.stretch_faces.shape[0] if bw else 0
    B = sc.bending.shape[0] if dih else 0
    ml = np.ascontiguousarray(sc.stretch_mu_lambda, np.float32) if sc.stretch_mu_lambda is not None and Fs else \
        np.tile(np.float32([sc.stretch_mu, sc.stretch_lambda]), (max(Fs, 1), 1))
    lib().orc_material_energy(sc.num_verts, _p(f4(x)), _p(f4(x_tilde)), _p(c(sc.mass, np.float32)),
                              _p(c(sc.pinned, np.uint8)), float(dt), float(sc.dirichlet), E,
                              _p(c(sc.edges, np.uint32)), _p(c(sc.rest_len, np.float32)),
                              _p(c(sc.spring_stiffness, np.float32) if sc.spring_stiffness is not None and E else
                                 np.full(max(E, 1), sc.spring_k, np.float32)), Fs, _p(c(sc.stretch_faces, np.uint32)),
                              _p(c(sc.stretch_dm_inv, np.float32)), _p(c(sc.stretch_area, np.float32)), _p(ml), B,
                              _p(c(sc.bending, np.uint32)), _p(c(sc.bending_rest_angle, np.float32)),
                              _p(c(sc.bending_hbar, np.float32)),
                              _p(c(sc.bending_stiffness, np.float32) if sc.bending_stiffness is not None and B else
                                 np.full(max(B, 1), sc.bending_k, np.float32)),
                              float(sc.bending_scaling), _p(out))
    return out
