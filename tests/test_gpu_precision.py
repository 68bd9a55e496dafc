"""Precision form: each FP32 / FP64-reduction result of the path against an all-FP64 computation of the same
algorithm on the same (FP32) inputs, with the errors printed (`pytest -s`) and bounded.

* PCG: K iterations of the GPU solve (FP32 dots and FP64 dots) against K iterations of the same block-Jacobi
  PCG in float64 (numpy/scipy) on the contact system of a folded cloth; the stop rules are switched off so
  that rounding alone separates the runs.
* Contact energy: the GPU's FP64 accumulation and a float32 accumulation of the same per-pair energies
  against a float64 evaluation and sum.
* ACCD step bound: see test_gpu_narrow.py (the FP64 form equals the all-FP64 oracle bit for bit)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from luisacomputesimulator_b200.linear import ConjugateGradientSolver, make_bsr
from oracle import oracle as O
from tests.gpu_util import dev, host
from tests.test_gpu_pcg import contact_system

pytestmark = pytest.mark.gpu


def _csr64(diag, A, B, n):
    rows, cols, vals = [], [], []
    d = np.asarray(diag, np.float64)[:, :, :3]  # 3 columns (float4) per row block, column-major
    for r in range(3):
        for c in range(3):
            rows.append(3 * np.arange(n) + r)
            cols.append(3 * np.arange(n) + c)
            vals.append(d[:, c, r])
    for m in (A, B):
        rp, col, val = m
        brow = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
        v = np.asarray(val, np.float64).reshape(-1, 3, 3)  # [k][c][r]
        for r in range(3):
            for c in range(3):
                rows.append(3 * brow + r)
                cols.append(3 * col.astype(np.int64) + c)
                vals.append(v[:, c, r])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(3 * n, 3 * n))


def _pcg64(M, diag, b, iters):
    n = b.shape[0]
    D = np.transpose(np.asarray(diag, np.float64)[:, :, :3], (0, 2, 1))
    Dinv = np.linalg.inv(D)
    x = np.zeros(3 * n)
    r = np.asarray(b, np.float64)[:, :3].reshape(-1).copy()
    p = np.zeros(3 * n)
    rz_old = 0.0
    for _ in range(iters):
        z = np.einsum("nij,nj->ni", Dinv, r.reshape(n, 3)).reshape(-1)
        rz = float(r @ z)
        beta = rz / rz_old if rz_old > 0 else 0.0
        rz_old = rz
        p = z + beta * p
        q = M @ p
        alpha = rz / float(p @ q)
        x += alpha * p
        r -= alpha * q
    return x.reshape(n, 3)


@pytest.mark.parametrize("iters", [10, 40])
def test_pcg_error_against_fp64(iters):
    sc, diag, A, B, b = contact_system()
    n = sc.num_verts
    x64 = _pcg64(_csr64(diag, A, B, n), diag, b, iters)
    err = {}
    for fp64 in (False, True):
        solver = ConjugateGradientSolver(n)
        x = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        bsr = lambda m: make_bsr(n, dev(m[0]), dev(m[1]), dev(m[2]))  # noqa: E731
        st = solver.device_solve(dev(diag), bsr(A), bsr(B), dev(b), x, max_iter=iters, rel_tol=0.0,
                                 abs_rz_tol=-1.0, check_every=1, fp64_dots=fp64)
        assert st["iterations"] == iters
        err[fp64] = float(np.linalg.norm(host(x)[:, :3] - x64) / np.linalg.norm(x64))
    print(f"\nPCG {iters} iterations: rel error vs all-FP64 run: FP32 dots {err[False]:.3e}, FP64 dots {err[True]:.3e}")
    assert err[False] < 1e-3 and err[True] < 1e-3


def test_contact_energy_error_against_fp64():
    from luisacomputesimulator_b200.collision import NarrowPhasesDetector
    from tests.gpu_util import SceneOnDevice
    from tests.test_gpu_narrow import _dcd
    sc, x0, det, got, want = _dcd("folded")
    D = SceneOnDevice(sc)
    det.reset_energy()
    det.compute_contact_energy(dev(x0), D.d_hat, D.offset)
    e_gpu = float(host(det.energy)[0])
    e64 = O.contact_energy(got, x0, sc.d_hat, sc.offset, fp64=True)
    e32 = O.contact_energy(got, x0, sc.d_hat, sc.offset, fp64=False)
    rel_gpu = abs(e_gpu - e64) / abs(e64)
    rel_32 = abs(e32 - e64) / abs(e64)
    print(f"\ncontact energy ({len(got)} pairs): rel error vs FP64 sum: GPU FP64 accumulation {rel_gpu:.3e}, "
          f"FP32 accumulation {rel_32:.3e}")
    assert rel_gpu <= 1e-5
    assert isinstance(det, NarrowPhasesDetector)
