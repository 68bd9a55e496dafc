"""Failure detection without a GPU fault: every failure is made on the host (a NaN written into the inputs, a tree
whose parent links were overwritten, a wait that no block satisfies) and each entry point must report it as a
status code, with the context still usable afterwards.

Reference behaviour restated: PCG stops on a NaN/Inf r.z (precond_cg.cpp:717-721), the Newton loop reports
a non-finite direction (newton_solver.cpp:3731-3737), fn_check_construction clears the healthy flag when a
child does not name its parent (lbvh.cpp:598-611, check_health lbvh.cpp:1033-1036), and waits are bounded
(wait_for_write, lbvh.cpp:62-82)."""
import numpy as np
import pytest
import torch

from luisacomputesimulator_b200 import _capi as A
from luisacomputesimulator_b200.collision import LBVH, stream
from luisacomputesimulator_b200.linear import ConjugateGradientSolver
from luisacomputesimulator_b200.newton import NewtonSolver
from oracle import oracle as O
from tests import scenarios as SC
from tests.gpu_util import dev
from tests.test_gpu_pcg import _dev_bsr, contact_system

pytestmark = pytest.mark.gpu


def _status_of(exc):
    return str(exc.value).split(":")[1].split()[0]


@pytest.mark.parametrize("mode", ["plain", "fused", "rows", "cg1"])
def test_pcg_reports_nan_right_hand_side(mode):
    sc, diag, Am, Bm, b = contact_system()
    n = sc.num_verts
    b = b.copy()
    saved = b[n // 3, 1]
    b[n // 3, 1] = np.nan
    solver = ConjugateGradientSolver(n)
    x = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(A.LcsError) as e:
        solver.device_solve(dev(diag), _dev_bsr(n, Am), _dev_bsr(n, Bm), dev(b), x, max_iter=100,
                            check_every=25 if mode == "plain" else 1, plain=mode == "plain", rows=mode == "rows",
                            single_reduction=mode == "cg1")
    assert _status_of(e) == "LCS_ERR_NAN"
    # the same solver with the finite right-hand side restored still solves
    b[n // 3, 1] = saved
    st = solver.device_solve(dev(diag), _dev_bsr(n, Am), _dev_bsr(n, Bm), dev(b), x, max_iter=500,
                             check_every=25 if mode == "plain" else 1, plain=mode == "plain", rows=mode == "rows",
                             single_reduction=mode == "cg1")
    assert st["status"] == 0 and st["rel_residual"] <= 1e-4


@pytest.mark.parametrize("plain", [False, True])
def test_newton_step_reports_a_nan_position(plain):
    """A NaN position uploaded from the host: the step returns LCS_ERR_NAN (the PCG's r.z is not finite) instead of
    applying a non-finite direction, and a later upload of a finite state steps normally."""
    sc, x = SC.cloth_touching_sphere(gap=5e-4, n=32)
    sc.x = x.copy()
    gpu = NewtonSolver(sc, plain=plain, single_reduction=not plain)
    st = gpu.step()
    assert st.status == 0
    good_x, good_v = gpu.positions(), gpu.velocities()
    bad = good_x.copy()
    bad[100, 1] = np.nan  # a free cloth vertex
    gpu.upload(bad, good_v)
    with pytest.raises(A.LcsError) as e:
        gpu.step()
    assert _status_of(e) == "LCS_ERR_NAN"
    gpu.upload(good_x, good_v)
    st = gpu.step()
    assert st.status == 0
    xn = gpu.positions()
    assert np.isfinite(xn).all()
    assert O.min_distance(sc, xn) > 0.0


def _face_tree():
    sc, x = SC.cloth_touching_sphere(gap=2e-3)
    xd = dev(x)
    t = LBVH(A.LCS_TREE_FACE, sc.faces.shape[0])
    t.reduce_face_tree_aabb(xd, dev(sc.faces))
    t.construct_tree()
    return t


def test_corrupted_parent_links_make_the_tree_unhealthy():
    t = _face_tree()
    assert t.check_health()
    data = t.device_data()
    parent = data["parent"]
    n = t.n
    saved = parent.clone()
    # leaf 7 (node n - 1 + 7) now names the root as its parent although the root's children are other nodes
    leaf = n - 1 + 7
    root_kids = data["children"][0].cpu().numpy()
    assert leaf not in root_kids
    parent[leaf] = 0
    torch.cuda.synchronize()
    t.check_construction()
    assert not t.check_health()
    # a swapped pair of inner-node parents is caught as well
    parent.copy_(saved)
    host_parent = saved.cpu().numpy()
    a = 1
    b = next(k for k in range(2, n - 1) if host_parent[k] != host_parent[a])
    pa, pb = int(host_parent[a]), int(host_parent[b])
    parent[a] = pb
    parent[b] = pa
    torch.cuda.synchronize()
    t.check_construction()
    assert not t.check_health()
    # restored links are healthy again, and so is a fresh build
    parent.copy_(saved)
    torch.cuda.synchronize()
    t.check_construction()
    assert t.check_health()
    t.construct_tree()
    assert t.check_health()


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_waits_run_out_and_report_timeout(which):
    """The slice-resident solve's reduction barrier (0) and neighbour-flag wait (1) with one block that never
    arrives: every other block gives up after a short poll limit and the call returns LCS_ERR_TIMEOUT."""
    lib = A.load()
    s = stream()
    assert lib.lcs_debug_pcg_wait(which, -1, 8, 1 << 20, s) == 0  # all blocks take part: the waits complete
    rc = lib.lcs_debug_pcg_wait(which, 3, 8, 1 << 12, s)
    assert A.STATUS[rc] == "LCS_ERR_TIMEOUT", A.STATUS.get(rc, rc)
    assert "ran out" in lib.lcs_last_error().decode()
    # the context is still usable: the same probe completes, and a solve runs
    assert lib.lcs_debug_pcg_wait(which, -1, 8, 1 << 20, s) == 0
    sc, diag, Am, Bm, b = contact_system()
    n = sc.num_verts
    x = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    st = ConjugateGradientSolver(n).device_solve(dev(diag), _dev_bsr(n, Am), _dev_bsr(n, Bm), dev(b), x,
                                                 max_iter=500, check_every=1, single_reduction=True)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-4


def test_wait_probe_rejects_bad_arguments():
    lib = A.load()
    s = stream()
    assert A.STATUS[lib.lcs_debug_pcg_wait(2, -1, 8, 16, s)] == "LCS_ERR_INVALID"
    assert A.STATUS[lib.lcs_debug_pcg_wait(0, -1, 64, 16, s)] == "LCS_ERR_INVALID"
    assert A.STATUS[lib.lcs_debug_pcg_wait(0, 9, 8, 16, s)] == "LCS_ERR_INVALID"
    assert A.STATUS[lib.lcs_debug_pcg_wait(0, -1, 8, 0, s)] == "LCS_ERR_INVALID"
