"""Host-side mirror of ConjugateGradientSolver (Solver/LinearSolver/precond_cg.h:17-71) and of
NewtonSolver::device_SpMV (newton_solver.cpp:3397-3427) over the C ABI."""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi as A
from .collision import ptr, stream


def make_bsr(n_rows, row_ptr, col, val):
    """lcs_bsr over CUDA tensors (row_ptr int32[n+1], col int32[nnzb], val float32[nnzb, 9])."""
    m = A.Bsr()
    m.n_rows = n_rows
    m.row_ptr = row_ptr.data_ptr()
    m.col = col.data_ptr()
    m.val = val.data_ptr()
    m._keep = (row_ptr, col, val)
    return m


def spmv(diag, A_bsr, B_bsr, x, y=None):
    n = x.shape[0]
    y = torch.empty_like(x) if y is None else y
    lib = A.load()
    A.check(lib.lcs_spmv(n, ptr(diag), C.byref(A_bsr) if A_bsr is not None else None,
                         C.byref(B_bsr) if B_bsr is not None else None, ptr(x), ptr(y), stream()), "spmv")
    return y


class ConjugateGradientSolver:
    """Block-Jacobi PCG with x0 = 0 (ConjugateGradientSolver::device_solve, precond_cg.cpp:626-771)."""

    def __init__(self, n):
        self.lib = A.load()
        self.n = int(n)
        h = C.c_void_p()
        A.check(self.lib.lcs_pcg_create(self.n, C.byref(h)), "pcg_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lcs_pcg_destroy(self.h)
            self.h = None

    def device_solve(self, diag, A_bsr, B_bsr, b, x, max_iter=100, rel_tol=1e-4, abs_rz_tol=1e-10, check_every=25,
                     fp64_dots=False, plain=False, rows=False, single_reduction=False):
        o = A.PcgOpts(max_iter, rel_tol, abs_rz_tol, check_every,
                      (A.LCS_PCG_FP64_DOTS if fp64_dots else 0) | (A.LCS_PCG_PLAIN if plain else 0) |
                      (A.LCS_PCG_ROWS if rows or single_reduction else 0) |
                      (A.LCS_PCG_SINGLE_REDUCTION if single_reduction else 0))
        st = A.PcgStats()
        A.check(self.lib.lcs_pcg_solve(self.h, ptr(diag), C.byref(A_bsr) if A_bsr is not None else None,
                                       C.byref(B_bsr) if B_bsr is not None else None, ptr(b), ptr(x), C.byref(o),
                                       C.byref(st), stream()), "pcg_solve")
        return dict(iterations=st.iterations, rel_residual=st.rel_residual, dot_rz=st.dot_rz, status=st.status)


def solve_batch(solver, row_offsets, diag, A_bsr, B_bsr, b, x, stats, active=None, max_iter=100, rel_tol=1e-4,
                abs_rz_tol=1e-10, check_every=1, fp64_dots=False, cluster=4):
    """Independent per-scene Jacobi-PCG solves in one launch (lcs_pcg_solve_batch).  row_offsets: CUDA
    int32 tensor of n_scenes + 1 offsets; stats: CUDA int32 tensor (n_scenes, 4) receiving lcs_pcg_stats."""
    import numpy as np
    lib = A.load()
    n_scenes = row_offsets.shape[0] - 1
    host_offs = np.ascontiguousarray(row_offsets.cpu().numpy().view(np.uint32))
    o = A.PcgOpts(max_iter, rel_tol, abs_rz_tol, check_every, A.LCS_PCG_FP64_DOTS if fp64_dots else 0)
    A.check(lib.lcs_pcg_solve_batch(solver.h, n_scenes, ptr(row_offsets), host_offs.ctypes.data_as(C.c_void_p),
                                    ptr(active), ptr(diag),
                                    C.byref(A_bsr) if A_bsr is not None else None,
                                    C.byref(B_bsr) if B_bsr is not None else None, ptr(b), ptr(x), C.byref(o),
                                    ptr(stats), cluster, stream()), "lcs_pcg_solve_batch")
