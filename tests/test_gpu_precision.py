"""Precision form: each FP32 / FP64-reduction result of the path against an all-FP64 computation of the same
algorithm on the same (FP32) inputs, with the errors printed (`pytest -s`) and bounded.

* PCG: K iterations of the GPU solve (FP32 dots and FP64 dots) against K iterations of the same block-Jacobi
  PCG in float64 (numpy/scipy) on the contact system of a folded cloth; the stop rules are switched off so
  that rounding alone separates the runs.
* Contact energy: the GPU's FP64 accumulation and a float32 accumulation of the same per-pair energies
  against a float64 evaluation and sum.
* ACCD step bound: see test_gpu_narrow.py (the FP64 form equals the all-FP64 oracle bit for bit).

The same on the 88,800-vertex tube at the benchmarked state (config 3): the system of the last Newton iteration
of the benchmarked step, its contact pairs and elastic energy, and its CCD candidates and step bound."""
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


# ----------------------------------------------------------------------------------------------- tube (config 3)
@pytest.fixture(scope="module")
def tube_iterate():
    from luisacomputesimulator_b200.newton import NewtonSolver
    from oracle import newton_cpu as N
    from tests import scenarios as SC
    from tests.test_gpu_tube import _oracle_contact_set
    sc, x, v, frame = SC.tube_state()
    gpu = NewtonSolver(sc, single_reduction=True)
    gpu.upload(x, v)
    gpu.set_frame(frame)
    assert gpu.step().status == 0
    x_iter, dx, x_tilde = gpu.last_iterate()
    _, _, pairs = _oracle_contact_set(sc, x_iter)
    b, diag, Am = N.material_fill(sc, N.MaterialPattern(sc), x_iter, x_tilde, sc.dt)
    b, diag = O.contact_grad_diag(pairs, sc.num_verts, b, diag)
    Bm = O.contact_offdiag_bsr(pairs, sc.num_verts)
    return dict(sc=sc, x_iter=x_iter, dx=dx, x_tilde=x_tilde, pairs=pairs, b=b, diag=diag, A=Am, B=Bm)


@pytest.mark.parametrize("iters", [25, 100])
def test_tube_pcg_error_against_fp64(tube_iterate, iters):
    """K iterations of the production solve (single reduction, slice-resident) with FP32 and with FP64 dot
    products against K iterations of the same PCG in float64 on the tube's 88,800-row system.  After 25
    iterations the three runs agree to ~1e-5; by the 100-iteration cap the FP32 matrix-vector products and
    vector updates have cost the FP32 runs their conjugacy and their true residual is ~3x the float64 run's,
    with or without FP64 dot products (measured 2.4e-3 and 2.9e-3 against 8.7e-4): the bound is 5x."""
    t = tube_iterate
    sc, diag, A, B, b = t["sc"], t["diag"], t["A"], t["B"], t["b"]
    n = sc.num_verts
    M = _csr64(diag, A, B, n)
    x64 = _pcg64(M, diag, b, iters)
    b64 = np.asarray(b, np.float64)[:, :3].reshape(-1)
    res = lambda y: float(np.linalg.norm(b64 - M @ y.reshape(-1)) / np.linalg.norm(b64))  # noqa: E731
    err, rr = {}, {}
    for fp64 in (False, True):
        solver = ConjugateGradientSolver(n)
        x = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        bsr = lambda m: make_bsr(n, dev(m[0]), dev(m[1]), dev(m[2]))  # noqa: E731
        st = solver.device_solve(dev(diag), bsr(A), bsr(B), dev(b), x, max_iter=iters, rel_tol=0.0,
                                 abs_rz_tol=-1.0, check_every=1, fp64_dots=fp64, single_reduction=True)
        assert st["iterations"] == iters
        xs = host(x)[:, :3].astype(np.float64)
        err[fp64] = float(np.linalg.norm(xs - x64) / np.linalg.norm(x64))
        rr[fp64] = res(xs)
    r64 = res(x64)
    print(f"\ntube PCG {iters} iterations: rel error vs all-FP64 run: FP32 dots {err[False]:.3e}, FP64 dots "
          f"{err[True]:.3e}; true rel residual: FP32 {rr[False]:.3e}, FP64 dots {rr[True]:.3e}, all-FP64 {r64:.3e}")
    assert err[False] < 5e-2 and err[True] < 5e-2
    assert rr[False] <= 5.0 * r64 + 1e-6 and rr[True] <= 5.0 * r64 + 1e-6


def test_tube_energy_sums_against_fp64(tube_iterate):
    """The line search's sums on the tube: the barrier energy of the contact pairs and the elastic + inertia
    energy, accumulated in FP64 on the GPU, against the oracle's float64 sums (and the FP32 accumulation the
    reference does)."""
    import ctypes as C

    from luisacomputesimulator_b200 import _capi as A
    from luisacomputesimulator_b200.collision import ptr, stream
    t = tube_iterate
    sc, x, pairs = t["sc"], t["x_iter"], t["pairs"]
    lib = A.load()
    dp = dev(np.ascontiguousarray(pairs).view(np.uint32).reshape(len(pairs), -1))
    cnt = dev(np.array([len(pairs)], np.uint32))
    xd, dh, off = dev(x), dev(sc.d_hat), dev(sc.offset)  # kept alive across the call
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    A.check(lib.lcs_contact_energy(ptr(dp), ptr(cnt), len(pairs), ptr(xd), ptr(dh), ptr(off), ptr(out), stream()),
            "lcs_contact_energy")
    e_gpu = float(host(out)[0])
    e64 = O.contact_energy(pairs, x, sc.d_hat, sc.offset, fp64=True)
    e32 = O.contact_energy(pairs, x, sc.d_hat, sc.offset, fp64=False)
    rel_gpu, rel_32 = abs(e_gpu - e64) / abs(e64), abs(e32 - e64) / abs(e64)
    # elastic + inertia (BW98 stretch, dihedral bending, inertia with the Dirichlet term), FP64 sums
    from tests.test_gpu_material import _cloth_elements
    m, keep = _cloth_elements(sc, x, t["x_tilde"])
    mo = torch.zeros(4, dtype=torch.float64, device="cuda")
    A.check(lib.lcs_material_energy(C.byref(m), ptr(keep["x"]), ptr(keep["xt"]), sc.dt, sc.dirichlet, ptr(mo),
                                    stream()), "lcs_material_energy")
    got = host(mo)
    want = O.material_energy(sc, x, t["x_tilde"], sc.dt)
    rel_m = float(np.abs(got - want).max() / np.abs(want).max())
    print(f"\ntube contact energy ({len(pairs)} pairs): rel error vs FP64 sum: GPU FP64 accumulation {rel_gpu:.3e}, "
          f"FP32 accumulation {rel_32:.3e}; material energy terms {got}: rel error {rel_m:.3e}")
    assert rel_gpu <= 1e-5 and rel_m <= 1e-5


def test_tube_step_bound_against_fp64(tube_iterate):
    """The CCD step bound along the last iteration's direction, lengthened four times so that contacts bound it
    (the direction itself is collision-free): per-pair TOI of the FP32 ACCD and of the precision form (whole
    iteration in FP64, TOI rounded toward zero) against the all-FP64 oracle ACCD on the tube's candidates; the
    precision form never exceeds it."""
    from luisacomputesimulator_b200.collision import NarrowPhasesDetector
    from tests.gpu_util import SceneOnDevice
    from tests.test_gpu_narrow import _load
    t = tube_iterate
    sc, x0, dx = t["sc"], t["x_iter"], t["dx"]
    x1 = x0.copy()
    x1[:, :3] = x0[:, :3] + np.float32(4.0) * dx[:, :3]
    tf = O.lbvh_build(O.TREE_FACE, x0, sc.faces, sc.num_verts)
    te = O.lbvh_build(O.TREE_EDGE, x0, sc.edges, sc.num_verts)
    O.lbvh_refit(tf, x0, x1, sc.faces, sc.offset)
    O.lbvh_refit(te, x0, x1, sc.edges, sc.offset)
    vf, _ = O.lbvh_query_vf(tf, x0, x1, sc.d_hat, sc.offset)
    ee, _ = O.lbvh_query_ee(te, x0, x1, sc.edges, sc.d_hat, sc.offset)
    want = {"vf": O.ccd_f64(False, vf, x0, x1, sc.faces, sc.body, sc.offset),
            "ee": O.ccd_f64(True, ee, x0, x1, sc.edges, sc.body, sc.offset)}
    g64 = min(want["vf"].min(initial=1.25), want["ee"].min(initial=1.25)) / 1.25
    assert g64 < 1.0 / 1.25  # contacts do bound this direction
    D = SceneOnDevice(sc)
    err, glob = {}, {}
    for fp64 in (False, True):  # the FP32 ACCD, the precision form (LCS_CCD_FP64)
        det = NarrowPhasesDetector(sc.num_verts, sc.edges.shape[0])
        _load(det, vf, ee)
        tvf = torch.zeros(det.cap_vf, dtype=torch.float32, device="cuda")
        tee = torch.zeros(det.cap_ee, dtype=torch.float32, device="cuda")
        det.reset_toi()
        det.vf_ccd_query(dev(x0), dev(x1), D.faces, D.body, D.offset, tvf, fp64=fp64)
        det.ee_ccd_query(dev(x0), dev(x1), D.edges, D.body, D.offset, tee, fp64=fp64)
        torch.cuda.synchronize()
        got = {"vf": host(tvf)[: len(vf)].astype(np.float64), "ee": host(tee)[: len(ee)].astype(np.float64)}
        err[fp64] = max(float(np.max(np.abs(got[k] - want[k]) / want[k], initial=0.0)) for k in got)
        glob[fp64] = float(host(det.toi)[0])
        if fp64:
            assert all((got[k] <= want[k]).all() for k in got)  # rounded toward zero: never above
    print(f"\ntube step bound ({len(vf)} VF + {len(ee)} EE candidates, 4 x the last direction): all-FP64 {g64:.9g}; "
          f"FP32 {glob[False]:.9g}, FP64 form {glob[True]:.9g}; largest per-pair rel error: FP32 {err[False]:.2e}, "
          f"FP64 form {err[True]:.2e}")
    assert err[True] <= 1e-6
    # the precision form's bound: the smallest FP64 TOI rounded toward zero, divided by 1.25 in float as the
    # reference divides it (toi / line_search_max_t)
    rz = []
    for k in want:
        f = want[k].astype(np.float32)
        f = np.where(f.astype(np.float64) > want[k], np.nextafter(f, np.float32(-np.inf)), f)
        rz.append(f.min(initial=np.float32(1.25)))
    assert glob[True] == float(np.float32(min(rz)) / np.float32(1.25))
    assert abs(glob[False] - g64) <= 1e-6 * g64  # the FP32 step bound itself
