"""Newton loop on the GPU: one iteration against the CPU restatement from the same contact-rich
state, plain vs fused agreement, and trajectories that stay intersection-free."""
import numpy as np
import pytest

from luisacomputesimulator_b200 import scenes as S
from luisacomputesimulator_b200.newton import NewtonSolver
from oracle import newton_cpu as N
from oracle import oracle as O
from tests import scenarios as SC

pytestmark = pytest.mark.gpu


def touching_scene(n=32, gap=5e-4):
    sc, x = SC.cloth_touching_sphere(gap=gap, n=n)
    sc.x = x.copy()  # start (and rest) on the sphere, inside d_hat
    return sc


def _predict(sc):
    x = sc.x.copy()
    xt = x.copy().astype(np.float32)
    free = ~sc.pinned.astype(bool)
    g = np.asarray(sc.gravity, np.float32)
    # v = 0: x_tilde = x + dt * (dt * g) for free vertices, the rest target for pinned ones
    xt[free, :3] = x[free, :3] + np.float32(sc.dt) * (np.float32(sc.dt) * g)
    return x, xt


def test_one_newton_iteration_matches_cpu_restatement():
    sc = touching_scene()
    gpu = NewtonSolver(sc, plain=True, nonlinear_iters=1, pcg_check_every=25)
    st = gpu.step()
    assert st.newton_iters == 1
    assert st.contact_pairs > 0
    xg = gpu.positions()
    x0, xt = _predict(sc)
    pat = N.MaterialPattern(sc)
    xc, toi, pst, cnt = N.newton_iteration(sc, x0, xt, sc.dt, pattern=pat)
    assert cnt["pairs"] == st.contact_pairs
    assert st.vf_candidates == cnt["vf"] and st.ee_candidates == cnt["ee"]
    dx_scale = np.abs(xc[:, :3] - x0[:, :3]).max()
    np.testing.assert_allclose(xg[:, :3], xc[:, :3], rtol=0, atol=2e-3 * dx_scale + 1e-7)
    assert abs(st.last_toi - toi) <= 1e-3 * toi + 1e-6


@pytest.mark.parametrize("fp64,cg1,gm", [(False, False, False), (True, False, False), (False, True, False),
                                         (False, True, True)])
def test_drop_stays_intersection_free(fp64, cg1, gm):
    # cloth rows first, sphere rows after: the contacts couple rows of distant blocks of the
    # slice-resident solve (its dependency mask beyond the neighbouring blocks)
    sc = S.cloth_on_sphere(n=32)
    gpu = NewtonSolver(sc, fp64=fp64, single_reduction=cg1, global_matrix=gm)
    assert gpu.pcg_kind() == (("cg1" if gm else "cg1-res") if cg1 else "rows")
    d0 = O.min_distance(sc, sc.x)
    for k in range(40):
        st = gpu.step()
        assert st.status == 0
        if k % 10 == 9:
            x = gpu.positions()
            assert np.isfinite(x).all()
            assert O.min_distance(sc, x) > 0.0
    x = gpu.positions()
    assert x[: 32 * 32, 1].min() < sc.x[: 32 * 32, 1].min()  # the cloth did fall
    assert O.min_distance(sc, x) > 0.0 and d0 > 0.0


@pytest.mark.parametrize("cg1", [False, True])
def test_plain_and_fused_agree_on_a_step(cg1):
    sc = touching_scene()
    a = NewtonSolver(sc, plain=True, pcg_check_every=1)
    b = NewtonSolver(sc, plain=False, single_reduction=cg1)
    sa, sb = a.step(), b.step()
    assert sa.newton_iters == sb.newton_iters
    xa, xb = a.positions(), b.positions()
    scale = np.abs(xa[:, :3] - sc.x[:, :3]).max()
    np.testing.assert_allclose(xa[:, :3], xb[:, :3], rtol=0, atol=5e-3 * scale + 1e-7)


def test_twisted_tube_steps_small():
    # a reduced tube (60 x 60) through the full step path, every mode
    for plain, cg1 in ((False, False), (False, True), (True, False)):
        sc = S.twisted_tube(60, 60)
        gpu = NewtonSolver(sc, plain=plain, single_reduction=cg1)
        for _ in range(5):
            st = gpu.step()
            assert 1 <= st.newton_iters <= 100  # the small-step rule may end the loop early
        x = gpu.positions()
        assert np.isfinite(x).all()
        assert O.min_distance(sc, x) > 0.0


def test_slice_resident_pcg_matches_the_global_form_on_the_tube():
    """The 88,800-row tube at a twisted, self-touching state: one step with the slice-resident solve
    (one block per SM, leading matrix groups in shared memory, neighbour-only publication waits) and
    one with the 256-row-block form that reads the matrix from L2.  Same summation order per row, so
    the steps agree to rounding of the grid-wide dot products."""
    sc, x = SC.twisted_tube_state(angle=1.2)
    out = {}
    for gm in (False, True):
        gpu = NewtonSolver(sc, single_reduction=True, global_matrix=gm)
        assert gpu.pcg_kind() == ("cg1" if gm else "cg1-res")
        st = gpu.step_host(x_in=x.copy())
        assert st.status == 0
        out[gm] = (gpu.positions(), st.pcg_iters, st.newton_iters)
    (xa, ia, na), (xb, ib, nb) = out[False], out[True]
    assert na == nb and abs(ia - ib) <= 2 * na
    scale = np.abs(xb[:, :3] - x[:, :3]).max()
    np.testing.assert_allclose(xa[:, :3], xb[:, :3], rtol=0, atol=1e-3 * scale + 1e-7)


def test_first_iteration_dcd_lists_filtered_across_steps_equal_a_traversal():
    """From the second step on, the first Newton iteration's DCD lists are the previous step's last CCD lists
    filtered at the step-start positions.  With one Newton iteration per step, every step's reported DCD
    candidate and pair counts are those of its first iteration: they must equal the oracle's static query and
    barrier pairs at the positions the step started from."""
    sc, x = SC.folded_cloth(n=32, gap=4e-4)
    gpu = NewtonSolver(sc, single_reduction=True, nonlinear_iters=1)
    st = gpu.step_host(x_in=x)
    checked = 0
    for _ in range(8):
        x0 = gpu.positions()
        st = gpu.step()
        assert st.status == 0
        if st.newton_iters != 1:
            continue
        tf = O.lbvh_build(O.TREE_FACE, x0, sc.faces, sc.num_verts)
        te = O.lbvh_build(O.TREE_EDGE, x0, sc.edges, sc.num_verts)
        O.lbvh_refit(tf, x0, x0, sc.faces, sc.offset)
        O.lbvh_refit(te, x0, x0, sc.edges, sc.offset)
        vf, n_vf = O.lbvh_query_vf(tf, x0, x0, sc.d_hat, sc.offset)
        ee, n_ee = O.lbvh_query_ee(te, x0, x0, sc.edges, sc.d_hat, sc.offset)
        pairs = len(O.dcd_vf(vf, x0, sc.faces, sc.body, sc.vert_area, sc.face_area, sc.d_hat, sc.offset, sc.kappa)) + \
            len(O.dcd_ee(ee, x0, sc.edges, sc.body, sc.edge_area, sc.d_hat, sc.offset, sc.kappa))
        assert (st.vf_candidates, st.ee_candidates) == (n_vf, n_ee)
        assert st.contact_pairs == pairs
        checked += 1
    assert checked >= 4


@pytest.mark.parametrize("plain", [True, False])
def test_c1_ten_steps_follow_the_cpu_restatement(plain):
    """Config 1 as configured (64 x 64 cloth dropped from 5 cm onto the pinned 2,562-vertex icosphere, dt 1/60,
    10 steps from rest).  Every GPU step is compared with the CPU restatement's time step from the same state
    (the GPU's state before the step): the first iteration's DCD candidates and contact pairs are equal (same
    positions), the Newton iteration counts are equal, and the new positions agree within 1e-3 of the step's
    motion (the PCG solves run to 1e-4 or to the 100-iteration cap, where FP32 rounding of different summation
    orders separates the iterates; measured up to 1.6e-4); the cloth stays intersection-free."""
    sc = S.cloth_on_sphere(n=64)
    gpu = NewtonSolver(sc, plain=plain, single_reduction=not plain)
    pat = N.MaterialPattern(sc)
    worst = 0.0
    touched = 0
    for k in range(10):
        xk, vk = gpu.positions(), gpu.velocities()
        st = gpu.step()
        assert st.status == 0
        log = gpu.iteration_log()
        xg = gpu.positions()
        xo, vo, recs = N.time_step(sc, xk, vk, k, pattern=pat, pcg_check_every=25 if plain else 1)
        assert (log[0]["vf_candidates"], log[0]["ee_candidates"], log[0]["contact_pairs"]) == \
            (recs[0]["vf"], recs[0]["ee"], recs[0]["pairs"])
        assert len(log) == len(recs)
        touched += log[0]["contact_pairs"] > 0
        motion = float(np.abs(xo[:, :3] - xk[:, :3]).max())
        dev_ = float(np.abs(xg[:, :3] - xo[:, :3]).max()) / motion
        worst = max(worst, dev_)
        assert dev_ <= 1e-3, (k, dev_)
        if k % 5 == 4:
            assert O.min_distance(sc, xg) > 0.0
    print(f"C1 ({'plain' if plain else 'fused'}): largest deviation {worst:.2e} of the step's motion; "
          f"{touched} steps with contact pairs")
    assert touched >= 2  # the cloth reached the sphere


def test_floor_ccd_bounds_the_step_like_the_reference():
    """fn_gound_collision_ccd: a cloth falling fast onto the floor (floor on, y = 0).  The step bound of the GPU's
    iteration equals the reference rule evaluated by the oracle on the GPU's own iterate and direction."""
    cx, cf = S.cloth_grid(32, 32, 0.01, origin=(0.0, 0.01, 0.0), jitter=1e-4, seed=3)
    sc = S.assemble("cloth_over_floor", [S.MeshPart(cx, cf, np.zeros(cx.shape[0], bool))], dt=1 / 60,
                    gravity=(0, -9.8, 0), kappa=1e7)
    v = np.zeros_like(sc.x)
    v[:, 1] = -2.0
    for plain in (False, True):
        gpu = NewtonSolver(sc, plain=plain, single_reduction=not plain, use_floor=True, floor_y=0.0,
                           nonlinear_iters=1)
        gpu.upload(sc.x, v)
        st = gpu.step()
        assert st.status == 0
        x_iter, dx, _ = gpu.last_iterate()
        x1 = x_iter.copy()
        x1[:, :3] = x_iter[:, :3] + dx[:, :3]
        floor = N.floor_ccd(x_iter, x1, sc.offset, sc.pinned, 0.0)
        assert floor < 1.0  # the unconstrained direction goes through the floor
        tf = O.lbvh_build(O.TREE_FACE, x_iter, sc.faces, sc.num_verts)
        te = O.lbvh_build(O.TREE_EDGE, x_iter, sc.edges, sc.num_verts)
        O.lbvh_refit(tf, x_iter, x1, sc.faces, sc.offset)
        O.lbvh_refit(te, x_iter, x1, sc.edges, sc.offset)
        cvf, _ = O.lbvh_query_vf(tf, x_iter, x1, sc.d_hat, sc.offset)
        cee, _ = O.lbvh_query_ee(te, x_iter, x1, sc.edges, sc.d_hat, sc.offset)
        g1, _ = O.ccd_vf(cvf, x_iter, x1, sc.faces, sc.body, sc.offset, per_pair=False)
        g2, _ = O.ccd_ee(cee, x_iter, x1, sc.edges, sc.body, sc.offset, per_pair=False)
        want = min(floor, g1, g2)
        got = gpu.iteration_log()[-1]["toi"]
        assert got <= want and abs(got - want) <= 1e-6 * want, (plain, got, want)
        x = gpu.positions()
        assert (x[:, 1] - sc.offset > 0.0).all()  # nothing below the floor


def test_deterministic_single_scene_repeats_bit_for_bit():
    """LCS_NEWTON_DETERMINISTIC on one scene (slice-resident PCG): two runs of 30 contact steps of the cloth
    falling on the sphere give the same bits.  The atomic form adds the same terms in another order: after the
    first step the two agree to 1e-3 of the step's motion (measured 1.4e-4 after the step's capped PCG solves;
    later contact steps amplify such rounding, as two atomic runs show)."""
    sc = S.cloth_on_sphere(n=32)
    runs = [NewtonSolver(sc, single_reduction=True, deterministic=True) for _ in range(2)]
    atomic = NewtonSolver(sc, single_reduction=True)
    assert atomic.step().status == 0
    pairs = 0
    for k in range(30):
        for g in runs:
            st = g.step()
            assert st.status == 0
            pairs = max(pairs, st.contact_pairs)
        if k == 0:
            xd, xc = runs[0].positions(), atomic.positions()
            scale = np.abs(xd[:, :3] - sc.x[:, :3]).max()
            assert scale > 0
            assert np.abs(xc[:, :3] - xd[:, :3]).max() <= 1e-3 * scale
    assert pairs > 0
    xa, xb = runs[0].positions(), runs[1].positions()
    np.testing.assert_array_equal(xa, xb)
    np.testing.assert_array_equal(runs[0].velocities(), runs[1].velocities())
    assert O.min_distance(sc, xa) > 0.0


def test_deterministic_mode_refuses_affine_bodies():
    from luisacomputesimulator_b200 import _capi as A
    sc = S.cloth_box_scene(400, 3)
    with pytest.raises(A.LcsError):
        NewtonSolver(sc, deterministic=True)
