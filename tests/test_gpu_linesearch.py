"""Energy line search (LCS_NEWTON_ENERGY_LINESEARCH, the reference's use_energy_linesearch,
Solver/SimulationSolver/newton_solver.cpp:3790-3834) against the oracle's decision.

After one Newton iteration the test reads the iteration's start positions, direction and inertial
target back, rebuilds the iteration-start contact pairs and the energies E(toi / 2^j) with the
oracle (inertia, BW98 stretch, dihedral bending, barrier), and checks that the device accepted the
first step length with E < E(0) + Epsilon -- the reference's rule -- unless that energy lies within
rounding of the threshold.  The fused loop (several step lengths per launch, decided on the device)
and the plain loop (one step length per host round trip) must take the same halvings."""
import numpy as np
import pytest

from luisacomputesimulator_b200.newton import NewtonSolver
from oracle import oracle as O
from tests import scenarios as SC

pytestmark = pytest.mark.gpu

EPS = float(np.float32(1.19209290e-7))


def _scene(gap=5e-4):
    sc, x = SC.cloth_touching_sphere(gap=gap, n=32)
    sc.x = x.copy()
    return sc


def _oracle_pairs(sc, x):
    tf = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    te = O.lbvh_build(O.TREE_EDGE, x, sc.edges, sc.num_verts)
    O.lbvh_refit(tf, x, x, sc.faces, sc.offset)
    O.lbvh_refit(te, x, x, sc.edges, sc.offset)
    vf, _ = O.lbvh_query_vf(tf, x, x, sc.d_hat, sc.offset)
    ee, _ = O.lbvh_query_ee(te, x, x, sc.edges, sc.d_hat, sc.offset)
    return np.concatenate([O.dcd_vf(vf, x, sc.faces, sc.body, sc.vert_area, sc.face_area, sc.d_hat, sc.offset,
                                    sc.kappa),
                           O.dcd_ee(ee, x, sc.edges, sc.body, sc.edge_area, sc.d_hat, sc.offset, sc.kappa)])


def _energy(sc, pairs, x, xt):
    return float(O.material_energy(sc, x, xt, sc.dt).sum()) + O.contact_energy(pairs, x, sc.d_hat, sc.offset)


def _velocity(sc, speed):
    v = np.zeros((sc.num_verts, 4), np.float32)
    v[~sc.pinned.astype(bool), 1] = -speed
    return v


def _oracle_halvings(sc, gpu, st):
    """The reference's decision for the last iteration, from the GPU's iterate: None on a tie."""
    x_it, dx, xt = gpu.last_iterate()
    pairs = _oracle_pairs(sc, x_it)
    toi = np.float32(st.last_toi)
    if np.linalg.norm(dx[:, :3], axis=1).max() < 1e-2 * sc.dt:  # small step: no search
        return 0, x_it, dx
    E0 = _energy(sc, pairs, x_it, xt)
    alpha = toi
    for j in range(21):
        xa = x_it.copy()
        xa[:, :3] = x_it[:, :3] + alpha * dx[:, :3]
        Ej = _energy(sc, pairs, xa, xt)
        if abs(Ej - (E0 + EPS)) <= 1e-7 * abs(E0):
            return None, x_it, dx
        if Ej < E0 + EPS:
            return j, x_it, dx
        alpha = np.float32(alpha / np.float32(2.0))
    raise AssertionError("no decrease within 20 halvings")


def _check_step(sc, gpu, st):
    want, x_it, dx = _oracle_halvings(sc, gpu, st)
    if want is None:
        return None
    toi = np.float32(st.last_toi)
    assert st.ls_halvings == want
    assert np.float32(st.last_alpha) == np.float32(toi / np.float32(2.0 ** want))
    np.testing.assert_array_equal(gpu.positions()[:, :3], x_it[:, :3] + np.float32(st.last_alpha) * dx[:, :3])
    return want


@pytest.mark.parametrize("speed", [0.0, 0.5, 2.0, 6.0])
def test_line_search_takes_the_oracle_step(speed):
    sc = _scene()
    gpu = NewtonSolver(sc, energy_linesearch=True, nonlinear_iters=1)
    st = gpu.step_host(x_in=sc.x.copy(), v_in=_velocity(sc, speed))
    assert st.status == 0 and st.newton_iters >= 1
    if st.newton_iters > 1:
        pytest.skip("more than one Newton iteration: the read-back holds the last one only")
    want = _check_step(sc, gpu, st)
    print(f"\nspeed {speed}: toi {st.last_toi:.4g}, halvings device {st.ls_halvings}, oracle {want}")


def test_line_search_halves_like_the_oracle_on_a_stiff_fold():
    """A folded cloth with 10^4 x the default bending stiffness: the Gauss-Newton bending Hessian
    underestimates the curvature and full steps raise the energy, so the search halves."""
    sc, x = SC.folded_cloth(n=32, gap=4e-4)
    sc.bending_k = 50.0
    sc.bending_stiffness[:] = 50.0  # the per-stencil stiffness takes precedence over the scalar
    gpu = NewtonSolver(sc, energy_linesearch=True, nonlinear_iters=1)
    st = gpu.step_host(x_in=x)
    halved, checked = 0, 0
    for k in range(12):
        if k:
            st = gpu.step()
        assert st.status == 0
        if st.newton_iters != 1:
            continue
        want = _check_step(sc, gpu, st)
        if want is not None:
            checked += 1
            halved += want > 0
    print(f"\nstiff fold: {checked} steps checked, {halved} with halvings")
    assert checked >= 6 and halved >= 1


def test_fused_and_plain_line_search_agree():
    sc = _scene()
    a = NewtonSolver(sc, energy_linesearch=True, plain=True, pcg_check_every=1)
    b = NewtonSolver(sc, energy_linesearch=True)
    v = _velocity(sc, 2.0)
    sa = a.step_host(x_in=sc.x.copy(), v_in=v)
    ha = (sa.newton_iters, sa.ls_halvings)
    sb = b.step_host(x_in=sc.x.copy(), v_in=v)
    hb = (sb.newton_iters, sb.ls_halvings)
    assert ha == hb
    xa, xb = a.positions(), b.positions()
    scale = np.abs(xa[:, :3] - sc.x[:, :3]).max()
    np.testing.assert_allclose(xa[:, :3], xb[:, :3], rtol=0, atol=5e-3 * scale + 1e-7)
    for _ in range(5):  # and the search keeps the drop intersection-free
        st = b.step()
        assert st.status == 0
    assert O.min_distance(sc, b.positions()) > 0.0
