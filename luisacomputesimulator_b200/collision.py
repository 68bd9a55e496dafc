"""Host-side mirror of the reference's collision-detector interface over the C ABI.

``LBVH`` keeps the method names of class LBVH (Solver/CollisionDetector/lbvh.h:166-229) and
``NarrowPhasesDetector`` those of class NarrowPhasesDetector
(Solver/CollisionDetector/narrow_phase.h:54-201), so code written against the reference
reads the same.  All tensors are CUDA tensors; the work runs on torch's current stream.
Errors raise ``LcsError`` with the library's status; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi as A

PAIR_BYTES = 48


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class _CudaArray:
    """A device buffer of the library seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr_, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr_), False),
                                         "version": 3, "strides": None}


def stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(t, dtype):
    assert t.is_cuda and t.dtype == dtype and t.is_contiguous(), f"expected contiguous CUDA {dtype}"
    return t


class Forest:
    """Per-scene LBVHs of many concatenated scenes in one set of arrays (batched solver).

    elem_offsets / vert_offsets: n_scenes + 1 prefix offsets of the scenes' elements and
    vertices.  Each scene's tree equals ``LBVH`` built on that scene alone."""

    def __init__(self, kind: int, elem_offsets, vert_offsets):
        import numpy as np
        self.lib = A.load()
        self.kind = kind
        eo = np.ascontiguousarray(elem_offsets, np.uint32)
        vo = np.ascontiguousarray(vert_offsets, np.uint32)
        self.elem_offsets, self.vert_offsets = eo, vo
        self.n_scenes = len(eo) - 1
        h = C.c_void_p()
        A.check(self.lib.lcs_forest_create(kind, self.n_scenes, eo.ctypes.data_as(C.c_void_p),
                                           vo.ctypes.data_as(C.c_void_p), C.byref(h)), "lcs_forest_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lcs_forest_destroy(self.h)
            self.h = None

    def build(self, x, elems):
        A.check(self.lib.lcs_forest_build(self.h, ptr(x), ptr(elems), stream()), "lcs_forest_build")

    def update_refit(self, thickness, x0, x1, elems):
        A.check(self.lib.lcs_forest_update_refit(self.h, ptr(thickness), ptr(x0), ptr(x1), ptr(elems), stream()),
                "lcs_forest_update_refit")

    def query_vf(self, x0, x1, vert_scene, d_hat, thickness, pairs, d_count):
        A.check(self.lib.lcs_forest_query_vf(self.h, ptr(x0), ptr(x1), x0.shape[0], ptr(vert_scene), ptr(d_hat),
                                             ptr(thickness), ptr(pairs), pairs.shape[0], ptr(d_count), stream()),
                "lcs_forest_query_vf")

    def query_ee(self, x0, x1, edges, d_hat, thickness, pairs, d_count):
        A.check(self.lib.lcs_forest_query_ee(self.h, ptr(x0), ptr(x1), ptr(edges), ptr(d_hat), ptr(thickness),
                                             ptr(pairs), pairs.shape[0], ptr(d_count), stream()), "lcs_forest_query_ee")

    def check_health(self):
        ok = C.c_int(0)
        A.check(self.lib.lcs_forest_health(self.h, C.byref(ok), stream()), "lcs_forest_health")
        return bool(ok.value)

    def query_tuning(self):
        """(threads per block, ms) of the traversal shape tuned on the first query (0 before it)."""
        t, ms = C.c_uint32(), C.c_float()
        A.check(self.lib.lcs_forest_query_tuning(self.h, C.byref(t), C.byref(ms)), "lcs_forest_query_tuning")
        return int(t.value), float(ms.value)

    def export_scene(self, scene):
        """(parent, children, object_idx, morton_sorted, sorted_get_original, node_aabb, global_aabb) of one
        scene's tree in the layout of LBVH.export (local ids)."""
        n = int(self.elem_offsets[scene + 1] - self.elem_offsets[scene])
        nn = 2 * n - 1
        d = lambda *shape, dt=torch.int32: torch.zeros(shape, dtype=dt, device="cuda")  # noqa: E731
        out = (d(nn), d(nn, 2), d(nn), d(n, dt=torch.int64), d(n), d(nn, 8, dt=torch.float32), d(6, dt=torch.float32))
        A.check(self.lib.lcs_forest_export_scene(self.h, scene, *[ptr(t) for t in out], stream()),
                "lcs_forest_export_scene")
        return out


class LBVH:
    """One LBVH over vertices, edges or faces (LbvhData + LBVH, lbvh.h:79-229)."""

    def __init__(self, kind: int, n_leaves: int):
        self.lib = A.load()
        self.kind, self.n = kind, int(n_leaves)
        h = C.c_void_p()
        A.check(self.lib.lcs_bvh_create(kind, self.n, C.byref(h)), "lcs_bvh_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lcs_bvh_destroy(self.h)
            self.h = None

    # -- construct (lbvh.cpp:939-998)
    def reduce_vert_tree_aabb(self, x):
        A.check(self.lib.lcs_bvh_reduce_aabb(self.h, ptr(x), None, x.shape[0], stream()), "reduce_aabb")

    def reduce_edge_tree_aabb(self, x, edges):
        A.check(self.lib.lcs_bvh_reduce_aabb(self.h, ptr(x), ptr(edges), x.shape[0], stream()), "reduce_aabb")

    def reduce_face_tree_aabb(self, x, faces):
        A.check(self.lib.lcs_bvh_reduce_aabb(self.h, ptr(x), ptr(faces), x.shape[0], stream()), "reduce_aabb")

    def construct_tree(self):
        A.check(self.lib.lcs_bvh_construct(self.h, stream()), "construct_tree")

    # -- refit (lbvh.cpp:1001-1045)
    def update_leaves(self, thickness, x0, x1, elems=None):
        A.check(self.lib.lcs_bvh_update_leaves(self.h, ptr(thickness), ptr(x0), ptr(x1), ptr(elems), stream()),
                "update_leaves")

    update_vert_tree_leave_aabb = update_leaves

    def update_edge_tree_leave_aabb(self, thickness, x0, x1, edges):
        self.update_leaves(thickness, x0, x1, edges)

    def update_face_tree_leave_aabb(self, thickness, x0, x1, faces):
        self.update_leaves(thickness, x0, x1, faces)

    def refit(self):
        A.check(self.lib.lcs_bvh_refit(self.h, stream()), "refit")

    def update_and_refit(self, thickness, x0, x1, elems=None):
        A.check(self.lib.lcs_bvh_update_refit(self.h, ptr(thickness), ptr(x0), ptr(x1), ptr(elems), stream()),
                "update_refit")

    def check_health(self) -> bool:
        ok = C.c_int(0)
        A.check(self.lib.lcs_bvh_health(self.h, C.byref(ok), stream()), "check_health")
        return bool(ok.value)

    def check_construction(self):
        """fn_check_construction (lbvh.cpp:598-611) on the tree as it is now; read the result with check_health."""
        A.check(self.lib.lcs_bvh_check_construction(self.h, stream()), "check_construction")

    def device_data(self):
        """The tree's device buffers (LbvhData layout) as int32 / int64 CUDA tensor views of the unsigned data:
        parent (2n-1,), children (2n-1, 2), morton_sorted (n,), sorted_get_original (n,).  Writing into them is
        the caller's business; run check_construction before any refit or query."""
        v = A.BvhDataView()
        A.check(self.lib.lcs_bvh_data(self.h, C.byref(v)), "lcs_bvh_data")
        n = int(v.n_leaves)
        view = lambda p, shape, typestr: torch.as_tensor(_CudaArray(p, shape, typestr), device="cuda")  # noqa: E731
        return {"parent": view(v.parent, (2 * n - 1,), "<i4"), "children": view(v.children, (2 * n - 1, 2), "<i4"),
                "morton_sorted": view(v.morton_sorted, (n,), "<i8"),
                "sorted_get_original": view(v.sorted_get_original, (n,), "<i4")}

    # -- queries (lbvh.cpp:1146-1192)
    def broad_phase_query_from_verts(self, x0, x1, count, pairs, d_hat, thickness):
        """Appends (vid, fid) pairs; `count` is a 1-element uint32 CUDA tensor (not reset here)."""
        A.check(self.lib.lcs_bvh_query_vf(self.h, ptr(x0), ptr(x1), x0.shape[0], ptr(d_hat), ptr(thickness),
                                          ptr(pairs), pairs.shape[0], ptr(count), stream()), "query_vf")

    def broad_phase_query_from_edges(self, x0, x1, edges, count, pairs, d_hat, thickness):
        A.check(self.lib.lcs_bvh_query_ee(self.h, ptr(x0), ptr(x1), ptr(edges), edges.shape[0], ptr(d_hat),
                                          ptr(thickness), ptr(pairs), pairs.shape[0], ptr(count), stream()),
                "query_ee")

    def broad_phase_query_from_edges_sym(self, x0, x1, edges, count, pairs, d_hat):
        """The set of broad_phase_query_from_edges for thickness 0 and one d_hat (a float) on every edge,
        each pair met once (no counterpart in the reference)."""
        A.check(self.lib.lcs_bvh_query_ee_sym(self.h, ptr(x0), ptr(x1), ptr(edges), float(d_hat), ptr(pairs),
                                              pairs.shape[0], ptr(count), stream()), "query_ee_sym")

    def export(self):
        """The tree in the reference's LbvhData layout (CUDA tensors)."""
        n = self.n
        nn = max(2 * n - 1, 1)
        dev = "cuda"
        out = dict(parent=torch.empty(nn, dtype=torch.int32, device=dev),
                   children=torch.empty((nn, 2), dtype=torch.int32, device=dev),
                   object_idx=torch.empty(nn, dtype=torch.int32, device=dev),
                   morton=torch.empty(max(n, 1), dtype=torch.int64, device=dev),
                   morton_sorted=torch.empty(max(n, 1), dtype=torch.int64, device=dev),
                   sorted_get_original=torch.empty(max(n, 1), dtype=torch.int32, device=dev),
                   node_aabb=torch.empty((nn, 8), dtype=torch.float32, device=dev),
                   global_aabb=torch.empty(6, dtype=torch.float32, device=dev))
        A.check(self.lib.lcs_bvh_export(self.h, ptr(out["parent"]), ptr(out["children"]), ptr(out["object_idx"]),
                                        ptr(out["morton"]), ptr(out["morton_sorted"]),
                                        ptr(out["sorted_get_original"]), ptr(out["node_aabb"]),
                                        ptr(out["global_aabb"]), stream()), "export")
        return out


class NarrowPhasesDetector:
    """CollisionData buffers + the narrow-phase entry points (narrow_phase.h:54-201).

    Capacities follow CollisionData::resize_collision_data_list (collision_data.h:445-485):
    4 x verts / 4 x edges broad-phase pairs, 2 x (verts + edges) contact pairs; they grow
    by doubling when a count comes back above capacity (NarrowPhasesDetector::resize_buffers).
    """

    def __init__(self, num_verts, num_edges, device="cuda"):
        self.lib = A.load()
        self.nv, self.ne = int(num_verts), int(num_edges)
        self.device = device
        self.cap_vf = max(4 * self.nv, 1024)
        self.cap_ee = max(4 * self.ne, 1024)
        self.cap_pairs = max(2 * (self.nv + self.ne), 1024)
        # counts: 0 vf broad, 1 ee broad, 2 narrow pairs, 3 spare
        self.counts = torch.zeros(4, dtype=torch.int32, device=device)
        self.toi = torch.ones(1, dtype=torch.float32, device=device)
        self.energy = torch.zeros(1, dtype=torch.float64, device=device)
        self._alloc()
        self.assembler = None

    def _alloc(self, which=("vf", "ee", "pairs")):
        if "vf" in which:
            self.broad_phase_list_vf = torch.zeros((self.cap_vf, 2), dtype=torch.int32, device=self.device)
        if "ee" in which:
            self.broad_phase_list_ee = torch.zeros((self.cap_ee, 2), dtype=torch.int32, device=self.device)
        if "pairs" in which:
            self.narrow_phase_list = torch.zeros((self.cap_pairs, 12), dtype=torch.int32, device=self.device)

    def count_view(self, k):
        return self.counts[k:k + 1]

    def reset_broadphase_count(self):
        self.counts[0:2].zero_()

    def reset_narrowphase_count(self):
        self.counts[2:3].zero_()

    def reset_toi(self):
        self.toi.fill_(1.0)

    def reset_energy(self):
        self.energy.zero_()

    def download_counts(self):
        return [int(v) for v in self.counts.cpu()]

    def resize_buffers(self):
        """Doubles whatever overflowed (NarrowPhasesDetector::resize_buffers, narrow_phase.cpp:61-95)."""
        c = self.download_counts()
        grew = []
        while c[0] > self.cap_vf:
            self.cap_vf *= 2
            grew.append("vf")
        while c[1] > self.cap_ee:
            self.cap_ee *= 2
            grew.append("ee")
        while c[2] > self.cap_pairs:
            self.cap_pairs *= 2
            grew.append("pairs")
            self.assembler = None
        if grew:
            self._alloc(set(grew))
        return bool(grew)

    # -- CCD (narrow_phase.cpp:293-740)
    def vf_ccd_query(self, x0, x1, faces, body, offset, toi_per_pair=None, fp64_final=False, fp64=False):
        flags = (A.LCS_CCD_FP64_FINAL if fp64_final else 0) | (A.LCS_CCD_FP64 if fp64 else 0)
        A.check(self.lib.lcs_ccd_vf(ptr(self.broad_phase_list_vf), ptr(self.count_view(0)), self.cap_vf, ptr(x0),
                                    ptr(x1), ptr(faces), ptr(body), ptr(offset), ptr(self.toi), ptr(toi_per_pair),
                                    flags, stream()), "ccd_vf")

    def ee_ccd_query(self, x0, x1, edges, body, offset, toi_per_pair=None, fp64_final=False, fp64=False):
        flags = (A.LCS_CCD_FP64_FINAL if fp64_final else 0) | (A.LCS_CCD_FP64 if fp64 else 0)
        A.check(self.lib.lcs_ccd_ee(ptr(self.broad_phase_list_ee), ptr(self.count_view(1)), self.cap_ee, ptr(x0),
                                    ptr(x1), ptr(edges), ptr(body), ptr(offset), ptr(self.toi), ptr(toi_per_pair),
                                    flags, stream()), "ccd_ee")

    def batched_ccd_query(self, is_ee, pairs, d_count, x0, x1, elems, body, offset, vert_scene, toi_per_scene,
                          fp64=False):
        """Batched scenes: the step bound of each candidate lowered into its own scene's bound."""
        A.check(self.lib.lcs_ccd_batch(int(bool(is_ee)), ptr(pairs), ptr(d_count), pairs.shape[0], ptr(x0), ptr(x1),
                                       ptr(elems), ptr(body), ptr(offset), ptr(vert_scene), ptr(toi_per_scene), None,
                                       A.LCS_CCD_FP64 if fp64 else 0, stream()), "lcs_ccd_batch")

    # -- DCD (narrow_phase.cpp:771-1249)
    def vf_dcd_query_repulsion(self, x, faces, body, vert_area, face_area, d_hat, offset, kappa):
        A.check(self.lib.lcs_dcd_vf(ptr(self.broad_phase_list_vf), ptr(self.count_view(0)), self.cap_vf, ptr(x),
                                    ptr(faces), ptr(body), ptr(vert_area), ptr(face_area), ptr(d_hat), ptr(offset),
                                    float(kappa), ptr(self.narrow_phase_list), self.cap_pairs,
                                    ptr(self.count_view(2)), stream()), "dcd_vf")

    def ee_dcd_query_repulsion(self, x, edges, body, edge_area, d_hat, offset, kappa):
        A.check(self.lib.lcs_dcd_ee(ptr(self.broad_phase_list_ee), ptr(self.count_view(1)), self.cap_ee, ptr(x),
                                    ptr(edges), ptr(body), ptr(edge_area), ptr(d_hat), ptr(offset), float(kappa),
                                    ptr(self.narrow_phase_list), self.cap_pairs, ptr(self.count_view(2)), stream()),
                "dcd_ee")

    # -- assembly (narrow_phase.cpp:1264-2362, 2550-2843)
    def device_perPair_evaluate_gradient_hessian(self, b, diag, abd=None):
        """abd: (body, model_x, body_dof) device tensors to remap rigid sides onto affine-body DOF slots."""
        if abd is None:
            A.check(self.lib.lcs_contact_grad_diag(ptr(self.narrow_phase_list), ptr(self.count_view(2)),
                                                   self.cap_pairs, ptr(b), ptr(diag), stream()), "grad_diag")
        else:
            v = abd_view(abd)
            A.check(self.lib.lcs_contact_grad_diag_abd(ptr(self.narrow_phase_list), ptr(self.count_view(2)),
                                                       self.cap_pairs, ptr(b), ptr(diag), C.byref(v), stream()),
                    "grad_diag_abd")

    def device_assemble_contact_triplet(self, abd=None):
        """Off-diagonal contact blocks as BSR; returns (lcs_bsr struct, nnzb device pointer)."""
        if self.assembler is None:
            h = C.c_void_p()
            create = self.lib.lcs_assembler_create_abd if abd is not None else self.lib.lcs_assembler_create
            A.check(create(self.nv, self.cap_pairs, C.byref(h)), "assembler_create")
            self.assembler = _Assembler(self.lib, h)
        if abd is None:
            A.check(self.lib.lcs_contact_offdiag_bsr(self.assembler.h, ptr(self.narrow_phase_list),
                                                     ptr(self.count_view(2)), self.cap_pairs, stream()), "offdiag_bsr")
        else:
            v = abd_view(abd)
            A.check(self.lib.lcs_contact_offdiag_bsr_abd(self.assembler.h, ptr(self.narrow_phase_list),
                                                         ptr(self.count_view(2)), self.cap_pairs, C.byref(v),
                                                         stream()), "offdiag_bsr_abd")
        return self.assembler.bsr()

    def compute_contact_energy(self, x, d_hat, offset):
        A.check(self.lib.lcs_contact_energy(ptr(self.narrow_phase_list), ptr(self.count_view(2)), self.cap_pairs,
                                            ptr(x), ptr(d_hat), ptr(offset), ptr(self.energy), stream()), "energy")


def abd_view(abd):
    """lcs_abd_view of (body, model_x, body_dof) device tensors."""
    body, model_x, body_dof = abd
    v = A.AbdView()
    v.body, v.model_x, v.body_dof = ptr(body), ptr(model_x), ptr(body_dof)
    return v


class _Assembler:
    def __init__(self, lib, h):
        self.lib, self.h = lib, h

    def bsr(self):
        m = A.Bsr()
        nnzb = C.c_void_p()
        A.check(self.lib.lcs_assembler_bsr(self.h, C.byref(m), C.byref(nnzb)), "assembler_bsr")
        return m, nnzb.value

    def export(self, n_rows, max_blocks):
        """(row_ptr, col, val) CUDA tensors of the assembled off-diagonal BSR."""
        rp = torch.empty(n_rows + 1, dtype=torch.int32, device="cuda")
        col = torch.empty(max(max_blocks, 1), dtype=torch.int32, device="cuda")
        val = torch.empty((max(max_blocks, 1), 9), dtype=torch.float32, device="cuda")
        nb = C.c_uint32(0)
        A.check(self.lib.lcs_assembler_export(self.h, ptr(rp), ptr(col), ptr(val), max_blocks, C.byref(nb), stream()),
                "assembler_export")
        return rp, col[: nb.value], val[: nb.value]

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lcs_assembler_destroy(self.h)
            self.h = None
