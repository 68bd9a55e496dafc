"""The 88,800-vertex twisted tube (config 2) through the fused Newton loop against the CPU restatement.

The state is the one the headline benchmark times: the tube after 56 steps of its run from rest, stepped by
the CPU restatement (tests/golden/tube88k_state.npz).  From the same positions the GPU's first Newton iteration
must find the oracle's DCD candidate sets and contact pairs (counts equal; the sets themselves are compared
bit for bit by the LBVH tests), its PCG solution must solve the oracle's system, and the step bound of any
iteration -- recomputed by the oracle from the GPU's own iterate and direction -- must match it within 1e-6
relative and never exceed it; the new positions are x_iter + toi dx exactly.  A 60-step run from rest must stay
intersection-free."""
import numpy as np
import pytest

from luisacomputesimulator_b200 import scenes as S
from luisacomputesimulator_b200.newton import NewtonSolver
from oracle import newton_cpu as N
from oracle import oracle as O
from tests import scenarios as SC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tube():
    sc, x, v, frame = SC.tube_state()
    return sc, x, v, frame, N.MaterialPattern(sc)


def _oracle_contact_set(sc, x):
    tf = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    te = O.lbvh_build(O.TREE_EDGE, x, sc.edges, sc.num_verts)
    O.lbvh_refit(tf, x, x, sc.faces, sc.offset)
    O.lbvh_refit(te, x, x, sc.edges, sc.offset)
    vf, n_vf = O.lbvh_query_vf(tf, x, x, sc.d_hat, sc.offset)
    ee, n_ee = O.lbvh_query_ee(te, x, x, sc.edges, sc.d_hat, sc.offset)
    pairs = np.concatenate([
        O.dcd_vf(vf, x, sc.faces, sc.body, sc.vert_area, sc.face_area, sc.d_hat, sc.offset, sc.kappa),
        O.dcd_ee(ee, x, sc.edges, sc.body, sc.edge_area, sc.d_hat, sc.offset, sc.kappa)])
    return n_vf, n_ee, pairs


def _ccd_bound(sc, x0, x1):
    tf = O.lbvh_build(O.TREE_FACE, x0, sc.faces, sc.num_verts)
    te = O.lbvh_build(O.TREE_EDGE, x0, sc.edges, sc.num_verts)
    O.lbvh_refit(tf, x0, x1, sc.faces, sc.offset)
    O.lbvh_refit(te, x0, x1, sc.edges, sc.offset)
    cvf, n_vf = O.lbvh_query_vf(tf, x0, x1, sc.d_hat, sc.offset)
    cee, n_ee = O.lbvh_query_ee(te, x0, x1, sc.edges, sc.d_hat, sc.offset)
    g1, _ = O.ccd_vf(cvf, x0, x1, sc.faces, sc.body, sc.offset, per_pair=False)
    g2, _ = O.ccd_ee(cee, x0, x1, sc.edges, sc.body, sc.offset, per_pair=False)
    return min(g1, g2), n_vf, n_ee


def test_first_iteration_from_the_tube_state_matches_the_oracle(tube):
    sc, x, v, frame, pat = tube
    gpu = NewtonSolver(sc, single_reduction=True, nonlinear_iters=1)
    gpu.upload(x, v)
    gpu.set_frame(frame)
    st = gpu.step()
    assert st.status == 0
    log = gpu.iteration_log()
    rec = log[0]
    # the oracle's first iteration of the same time step
    xt, _ = N.predict(sc, x, v, N.step_time(frame, sc.dt))
    n_vf, n_ee, pairs = _oracle_contact_set(sc, x)
    assert (rec["vf_candidates"], rec["ee_candidates"]) == (n_vf, n_ee)
    assert rec["contact_pairs"] == len(pairs) > 1000
    info = {}
    xc, toi, pst, cnt = N.newton_iteration(sc, x, xt, sc.dt, pattern=pat, pcg_check_every=1, info=info)
    assert (cnt["vf"], cnt["ee"], cnt["pairs"]) == (n_vf, n_ee, len(pairs))
    assert abs(rec["pcg_iters"] - pst["iterations"]) <= 1
    # the step bound of the last iterate, recomputed by the oracle from the GPU's iterate and direction
    x_iter, dx, x_tilde = gpu.last_iterate()
    rec = log[-1]
    toi_o, c_vf, c_ee = _ccd_bound(sc, x_iter, _stepped(x_iter, dx, 1.0))
    assert (rec["ccd_vf_candidates"], rec["ccd_ee_candidates"]) == (c_vf, c_ee)
    assert rec["toi"] <= toi_o and abs(rec["toi"] - toi_o) <= 1e-6 * toi_o
    np.testing.assert_array_equal(gpu.positions()[:, :3], _stepped(x_iter, dx, rec["toi"])[:, :3])
    # targets and prediction: the pinned rings' inertial targets agree to the rounding of cosf / sinf
    np.testing.assert_allclose(x_tilde[:, :3], xt[:, :3], rtol=0, atol=1e-6)
    assert st.newton_iters == 1, "the pinned rings reach their targets within 1e-3 in the first iteration"
    np.testing.assert_array_equal(x_iter, x)
    # both directions come from a one-iteration PCG solve: they agree to the rounding of its dot products
    scale = np.abs(info["dx"][:, :3]).max()
    np.testing.assert_allclose(dx[:, :3], info["dx"][:, :3], rtol=0, atol=1e-5 * scale)
    assert abs(rec["toi"] - toi) <= 1e-6 * toi


def _stepped(x0, dx, alpha):
    out = x0.copy()
    out[:, :3] = x0[:, :3] + np.float32(alpha) * dx[:, :3]
    return out


def test_the_benchmarked_step_matches_the_oracle_on_its_last_iterate(tube):
    """The full benchmarked time step (3 Newton iterations, PCG capped at 100): the last iteration's contact set,
    system, step bound and update against the oracle from the GPU's own iterate."""
    sc, x, v, frame, pat = tube
    gpu = NewtonSolver(sc, single_reduction=True)
    gpu.upload(x, v)
    gpu.set_frame(frame)
    st = gpu.step()
    assert st.status == 0 and st.newton_iters == 3
    log = gpu.iteration_log()
    assert len(log) == 3 and all(r["pcg_iters"] <= 100 for r in log)
    rec = log[-1]
    x_iter, dx, x_tilde = gpu.last_iterate()
    n_vf, n_ee, pairs = _oracle_contact_set(sc, x_iter)
    assert (rec["vf_candidates"], rec["ee_candidates"], rec["contact_pairs"]) == (n_vf, n_ee, len(pairs))
    # the GPU direction solves the oracle's system about as well as the oracle's own capped PCG: both are FP32
    # solves stopped at 100 iterations, which different rounding leaves a few times apart (measured 0.6x-1.3x)
    b, diag, Am = N.material_fill(sc, pat, x_iter, x_tilde, sc.dt)
    b, diag = O.contact_grad_diag(pairs, sc.num_verts, b, diag)
    Bm = O.contact_offdiag_bsr(pairs, sc.num_verts)
    ox, ost = O.pcg(diag, Am, Bm, b, max_iter=100, rel_tol=1e-4, check_every=1)
    nb = np.linalg.norm(b[:, :3].astype(np.float64))
    res = lambda y: np.linalg.norm(b[:, :3].astype(np.float64) - O.bsr_spmv(diag, Am, Bm, y)[:, :3]) / nb  # noqa: E731
    r_gpu, r_orc = res(dx), res(ox)
    print(f"true relative residual: GPU {r_gpu:.3e}, oracle {r_orc:.3e}; iterations {rec['pcg_iters']} vs "
          f"{ost['iterations']}")
    assert r_gpu <= 3.0 * r_orc + 1e-6
    toi_o, c_vf, c_ee = _ccd_bound(sc, x_iter, _stepped(x_iter, dx, 1.0))
    assert (rec["ccd_vf_candidates"], rec["ccd_ee_candidates"]) == (c_vf, c_ee)
    assert rec["toi"] <= toi_o and abs(rec["toi"] - toi_o) <= 1e-6 * toi_o
    np.testing.assert_array_equal(gpu.positions()[:, :3], _stepped(x_iter, dx, rec["toi"])[:, :3])
    assert O.min_distance(sc, gpu.positions()) > 0.0


def test_tube_run_from_rest_stays_intersection_free():
    """Config 2 as configured: 60 steps from rest (rings at -/+2 rad/s), minimum VF / EE distance > 0 every 10
    steps, contacts present by the end."""
    sc = S.twisted_tube(300, 296)
    gpu = NewtonSolver(sc, single_reduction=True)
    pairs = []
    for k in range(60):
        st = gpu.step()
        assert st.status == 0
        pairs.append(st.contact_pairs)
        if k % 10 == 9:
            x = gpu.positions()
            assert np.isfinite(x).all()
            d = O.min_distance(sc, x)
            print(f"step {k + 1}: min distance {d:.3e}, contact pairs {st.contact_pairs}")
            assert d > 0.0
    assert max(pairs[-10:]) > 1000
