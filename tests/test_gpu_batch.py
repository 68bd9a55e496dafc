"""Batched scenes: forests of per-scene LBVHs, per-scene CCD bounds and per-scene PCG against the oracle
run on each scene alone, and batched Newton trajectories that do not depend on the other scenes."""
import numpy as np
import pytest
import torch

from luisacomputesimulator_b200 import _capi as A
from luisacomputesimulator_b200 import scenes as S
from luisacomputesimulator_b200.collision import Forest, NarrowPhasesDetector
from luisacomputesimulator_b200.linear import ConjugateGradientSolver, make_bsr, solve_batch
from luisacomputesimulator_b200.newton import NewtonBatch
from oracle import oracle as O
from tests import scenarios as SC
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu


def _scenes():
    """Three scenes of different sizes, each with contact, and swept end positions."""
    out = []
    for k, (sc, x) in enumerate([SC.cloth_touching_sphere(gap=5e-4, n=24), SC.folded_cloth(n=32, gap=4e-4),
                                 SC.cloth_touching_sphere(gap=8e-4, n=40)]):
        out.append((sc, x, SC.random_motion(x, 1.5e-3, seed=20 + k)))
    return out


def _concat(items):
    """Concatenate scenes (indices shifted by the vertex offset) for the forest entry points."""
    vo, fo, eo = [0], [0], [0]
    xs, x1s, faces, edges, dh, off = [], [], [], [], [], []
    for sc, x, x1 in items:
        f = sc.faces.astype(np.uint32).copy()
        f[:, :3] += vo[-1]
        faces.append(f)
        edges.append(sc.edges.astype(np.uint32) + vo[-1])
        xs.append(x)
        x1s.append(x1)
        dh.append(sc.d_hat)
        off.append(sc.offset)
        vo.append(vo[-1] + sc.num_verts)
        fo.append(fo[-1] + sc.faces.shape[0])
        eo.append(eo[-1] + sc.edges.shape[0])
    vscene = np.concatenate([np.full(items[k][0].num_verts, k, np.uint32) for k in range(len(items))])
    return dict(vo=np.array(vo, np.uint32), fo=np.array(fo, np.uint32), eo=np.array(eo, np.uint32),
                x=np.concatenate(xs), x1=np.concatenate(x1s), faces=np.concatenate(faces),
                edges=np.concatenate(edges), d_hat=np.concatenate(dh), offset=np.concatenate(off), vscene=vscene)


@pytest.fixture(scope="module")
def batch():
    items = _scenes()
    return items, _concat(items)


def test_forest_update_before_build_is_refused(batch):
    """A forest's sorted order and slots come from its build: an update, query or export before it is refused
    (LCS_ERR_INVALID)."""
    items, c = batch
    f = Forest(O.TREE_FACE, c["fo"], c["vo"])
    xd, ed = dev(c["x"]), dev(c["faces"])
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.zeros((1024, 2), dtype=torch.int32, device="cuda")
    for call in (lambda: f.update_refit(dev(c["offset"]), xd, xd, ed), lambda: f.export_scene(0),
                 lambda: f.query_vf(xd, xd, dev(c["vscene"]), dev(c["d_hat"]), dev(c["offset"]), pairs, cnt)):
        with pytest.raises(A.LcsError, match="LCS_ERR_INVALID"):
            call()
    f.build(xd, ed)
    f.update_refit(dev(c["offset"]), xd, xd, ed)
    assert f.check_health()


@pytest.mark.parametrize("kind_name", ["face", "edge"])
def test_forest_trees_equal_standalone_oracle_trees(batch, kind_name):
    items, c = batch
    kind = O.TREE_FACE if kind_name == "face" else O.TREE_EDGE
    elems = c["faces"] if kind_name == "face" else c["edges"]
    offs = c["fo"] if kind_name == "face" else c["eo"]
    f = Forest(kind, offs, c["vo"])
    xd, x1d, ed = dev(c["x"]), dev(c["x1"]), dev(elems)
    f.build(xd, ed)
    f.update_refit(dev(c["offset"]), xd, x1d, ed)
    f.update_refit(dev(c["offset"]), xd, x1d, ed)  # twice: the arrival counters reset themselves
    assert f.check_health()
    for k, (sc, x, x1) in enumerate(items):
        own = sc.faces if kind_name == "face" else sc.edges
        t_o = O.lbvh_build(kind, x, own, sc.num_verts)
        O.lbvh_refit(t_o, x, x1, own, sc.offset)
        parent, children, object_idx, ms, sgo, aabb, g = f.export_scene(k)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(host(g), np.concatenate([t_o.gmin, t_o.gmax]))
        np.testing.assert_array_equal(host(ms, np.uint64), t_o.morton_sorted)
        np.testing.assert_array_equal(host(sgo, np.uint32), t_o.sorted_get_original)
        np.testing.assert_array_equal(host(parent, np.uint32), t_o.parent)
        np.testing.assert_array_equal(host(children, np.uint32), t_o.children)
        np.testing.assert_array_equal(host(object_idx, np.uint32), t_o.object_idx)
        got = host(aabb)
        np.testing.assert_array_equal(got[:, 0:3], t_o.node_aabb[:, 0:3])
        np.testing.assert_array_equal(got[:, 4:7], t_o.node_aabb[:, 4:7])


def test_forest_candidate_sets_equal_per_scene_oracle(batch):
    items, c = batch
    xd, x1d = dev(c["x"]), dev(c["x1"])
    ff = Forest(O.TREE_FACE, c["fo"], c["vo"])
    fe = Forest(O.TREE_EDGE, c["eo"], c["vo"])
    fd, edd, dh, off = dev(c["faces"]), dev(c["edges"]), dev(c["d_hat"]), dev(c["offset"])
    ff.build(xd, fd)
    fe.build(xd, edd)
    ff.update_refit(off, xd, x1d, fd)
    fe.update_refit(off, xd, x1d, edd)
    want_vf, want_ee = [], []
    for k, (sc, x, x1) in enumerate(items):
        tf = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
        O.lbvh_refit(tf, x, x1, sc.faces, sc.offset)
        vf, _ = O.lbvh_query_vf(tf, x, x1, sc.d_hat, sc.offset)
        te = O.lbvh_build(O.TREE_EDGE, x, sc.edges, sc.num_verts)
        O.lbvh_refit(te, x, x1, sc.edges, sc.offset)
        ee, _ = O.lbvh_query_ee(te, x, x1, sc.edges, sc.d_hat, sc.offset)
        want_vf.append(np.asarray(vf, np.int64).reshape(-1, 2) + np.array([c["vo"][k], c["fo"][k]]))
        want_ee.append(np.asarray(ee, np.int64).reshape(-1, 2) + c["eo"][k])
    want_vf, want_ee = np.concatenate(want_vf), np.concatenate(want_ee)
    # the first query of a forest tunes its launch shape (one run per shape, the count restored in between);
    # the second uses the tuned shape and appends behind the first: both must give the oracle's sets
    for q, want in (("vf", want_vf), ("ee", want_ee)):
        cnt = torch.full((1,), 5, dtype=torch.int32, device="cuda")  # appends start behind 5 earlier pairs
        pairs = torch.zeros((2 * len(want) + 64, 2), dtype=torch.int32, device="cuda")
        for rep in range(2):
            if q == "vf":
                ff.query_vf(xd, x1d, dev(c["vscene"]), dh, off, pairs, cnt)
            else:
                fe.query_ee(xd, x1d, edd, dh, off, pairs, cnt)
            n = int(host(cnt, np.uint32)[0])
            assert n == 5 + (rep + 1) * len(want)
            got = host(pairs, np.uint32)[5 + rep * len(want): n]
            np.testing.assert_array_equal(SC.sorted_pairs(got), SC.sorted_pairs(want))
        threads, ms = (ff if q == "vf" else fe).query_tuning()
        assert threads in (64, 128, 256) and ms > 0.0


@pytest.mark.parametrize("fp64", [False, True])
def test_batched_ccd_bounds_equal_single_scene_bounds(batch, fp64):
    items, c = batch
    body = dev(np.concatenate([sc.body for sc, _, _ in items]))
    xd, x1d, off = dev(c["x"]), dev(c["x1"]), dev(c["offset"])
    for q, elems in (("vf", c["faces"]), ("ee", c["edges"])):
        # candidates: the concatenation of each scene's oracle candidates
        cand, shift = [], []
        for k, (sc, x, x1) in enumerate(items):
            if q == "vf":
                t = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
                O.lbvh_refit(t, x, x1, sc.faces, sc.offset)
                p, _ = O.lbvh_query_vf(t, x, x1, sc.d_hat, sc.offset)
                shift.append(np.array([c["vo"][k], c["fo"][k]], np.int64))
            else:
                t = O.lbvh_build(O.TREE_EDGE, x, sc.edges, sc.num_verts)
                O.lbvh_refit(t, x, x1, sc.edges, sc.offset)
                p, _ = O.lbvh_query_ee(t, x, x1, sc.edges, sc.d_hat, sc.offset)
                shift.append(np.array([c["eo"][k], c["eo"][k]], np.int64))
            cand.append(np.asarray(p, np.int64).reshape(-1, 2))
        pairs = np.concatenate([cand[k] + shift[k] for k in range(len(items))]).astype(np.uint32)
        det = NarrowPhasesDetector(len(c["vscene"]), len(c["edges"]))
        toi = torch.ones(len(items), dtype=torch.float32, device="cuda")
        cnt = torch.tensor([len(pairs)], dtype=torch.int32, device="cuda")
        det.batched_ccd_query(q == "ee", dev(pairs), cnt, xd, x1d, dev(elems), body, off, dev(c["vscene"]), toi,
                              fp64=fp64)
        got = host(toi)
        for k, (sc, x, x1) in enumerate(items):
            fn = O.ccd_ee if q == "ee" else O.ccd_vf
            g, _ = fn(cand[k], x, x1, sc.edges if q == "ee" else sc.faces, sc.body, sc.offset, per_pair=False)
            if fp64:  # the FP64 iteration can differ from the FP32 one by about float precision
                assert abs(got[k] - g) <= 1e-6 * g
            else:
                assert got[k] == np.float32(g)


def _scene_system(sc, x):
    from tests.test_gpu_pcg import spring_system
    tf = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    O.lbvh_refit(tf, x, x, sc.faces, sc.offset)
    vf, _ = O.lbvh_query_vf(tf, x, x, sc.d_hat, sc.offset)
    te = O.lbvh_build(O.TREE_EDGE, x, sc.edges, sc.num_verts)
    O.lbvh_refit(te, x, x, sc.edges, sc.offset)
    ee, _ = O.lbvh_query_ee(te, x, x, sc.edges, sc.d_hat, sc.offset)
    pairs = np.concatenate([O.dcd_vf(vf, x, sc.faces, sc.body, sc.vert_area, sc.face_area, sc.d_hat, sc.offset,
                                     sc.kappa),
                            O.dcd_ee(ee, x, sc.edges, sc.body, sc.edge_area, sc.d_hat, sc.offset, sc.kappa)])
    diag, A = spring_system(sc, x)
    b = np.zeros((sc.num_verts, 4), np.float32)
    b, diag = O.contact_grad_diag(pairs, sc.num_verts, b, diag)
    b[:, :3] += np.random.default_rng(sc.num_verts).normal(0, 1e-3, (sc.num_verts, 3)).astype(np.float32)
    return diag, A, O.contact_offdiag_bsr(pairs, sc.num_verts), b


def _block_diag(mats, offs):
    rps, cols, vals = [], [], []
    base = 0
    for (rp, col, val), o in zip(mats, offs):
        rps.append(rp[:-1].astype(np.int64) + base)
        cols.append(col.astype(np.int64) + o)
        vals.append(val)
        base += len(col)
    rps.append(np.array([base]))
    return np.concatenate(rps).astype(np.uint32), np.concatenate(cols).astype(np.uint32), np.concatenate(vals)


@pytest.fixture(scope="module")
def systems(batch):
    items, c = batch
    return [_scene_system(sc, x) for sc, x, _ in items], c


def _solve(systems_c, which, cluster):
    systems, c = systems_c
    sel = [systems[k] for k in which]
    nv = [systems[k][3].shape[0] for k in which]
    offs = np.concatenate([[0], np.cumsum(nv)]).astype(np.uint32)
    n = int(offs[-1])
    diag = np.concatenate([s[0] for s in sel])
    b = np.concatenate([s[3] for s in sel])
    A = _block_diag([s[1] for s in sel], offs[:-1])
    B = _block_diag([s[2] for s in sel], offs[:-1])
    solver = ConjugateGradientSolver(n)
    x = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    stats = torch.zeros((len(which), 4), dtype=torch.int32, device="cuda")
    bsr = lambda m: make_bsr(n, dev(m[0]), dev(m[1]), dev(m[2]))  # noqa: E731
    solve_batch(solver, dev(offs), dev(diag), bsr(A), bsr(B), dev(b), x, stats, max_iter=300, rel_tol=1e-4,
                cluster=cluster)
    torch.cuda.synchronize()
    return host(x), offs, host(stats)


@pytest.mark.parametrize("cluster", [0, 1, 4, 16])
def test_batched_pcg_per_scene_matches_oracle_and_is_independent(systems, cluster):
    sysl, c = systems
    x, offs, stats = _solve(systems, [0, 1, 2], cluster)
    x_ref, _, _ = _solve(systems, [0, 1, 2], 2)
    np.testing.assert_array_equal(x, x_ref)  # the cluster size does not change any result
    for k, (diag, A, B, b) in enumerate(sysl):
        xs = x[offs[k]:offs[k + 1]]
        alone, _, st_alone = _solve(systems, [k], cluster)
        np.testing.assert_array_equal(xs, alone)  # alone == in the mix, bit for bit
        assert stats[k, 0] == st_alone[0, 0]
        ox, ost = O.pcg(diag, A, B, b, max_iter=300, rel_tol=1e-4, check_every=1)
        assert stats[k, 3] == 0 and ost["status"] == 0
        assert abs(int(stats[k, 0]) - ost["iterations"]) <= max(3, ost["iterations"] // 20 + 1)
        # the stop rules are the reference's (r.z < 1e-10 or |r| <= 1e-4 |r0|): the true residual of the
        # batched solve is within 1.5x of the oracle's own at its stop
        res = lambda xx: np.linalg.norm(b[:, :3].astype(np.float64) -  # noqa: E731
                                        O.bsr_spmv(diag, A, B, xx)[:, :3].astype(np.float64))
        assert res(xs) <= 1.5 * res(ox) + 1e-6 * np.linalg.norm(b[:, :3])
        np.testing.assert_allclose(xs[:, :3], ox[:, :3], rtol=0, atol=2e-3 * np.abs(ox).max())


def _drapes():
    return [S.random_cloth_scene(n, seed) for n, seed in ((400, 1), (900, 2), (1600, 3))]


def test_deterministic_batch_is_bit_identical_alone_and_in_mix():
    """LCS_NEWTON_DETERMINISTIC (the batch default): the cloth terms summed per row and per block in element
    order, the contact pairs sorted into a canonical order before their sums -- a scene's 8 contact steps are
    bit-identical in a mix of three, alone, and alone once more."""
    scs = _drapes()
    mix = NewtonBatch(scs, deterministic=True)
    alone = [NewtonBatch([sc], deterministic=True) for sc in scs]
    again = [NewtonBatch([sc], deterministic=True) for sc in scs]
    assert mix.deterministic
    pairs = 0
    for _ in range(8):
        st = mix.step()
        assert st.status == 0
        pairs = max(pairs, st.contact_pairs)
        for a in alone + again:
            assert a.step().status == 0
    assert pairs > 0, "the drapes touch their colliders"
    for k, sc in enumerate(scs):
        xm, xa, xb = mix.positions(k), alone[k].positions(0), again[k].positions(0)
        np.testing.assert_array_equal(xm, xa)
        np.testing.assert_array_equal(xb, xa)
        np.testing.assert_array_equal(mix.velocities(k), alone[k].velocities(0))
        assert np.abs(xa[:, :3] - sc.x[:, :3]).max() > 0
        assert O.min_distance(sc, xm) > 0.0


def test_batched_newton_alone_equals_in_mix_and_stays_intersection_free():
    """The same with float atomics (deterministic=False): within the run-to-run spread of the atomics."""
    scs = _drapes()
    mix = NewtonBatch(scs, deterministic=False)
    alone = [NewtonBatch([sc], deterministic=False) for sc in scs]
    again = [NewtonBatch([sc], deterministic=False) for sc in scs]  # the same scene alone once more: the run-to-run spread
    for _ in range(8):
        st = mix.step()
        assert st.status == 0
        for a in alone + again:
            a.step()
    for k, sc in enumerate(scs):
        xm, xa, xb = mix.positions(k), alone[k].positions(0), again[k].positions(0)
        assert np.isfinite(xm).all()
        assert mix.scene_stats(k).newton_iters == alone[k].scene_stats(0).newton_iters
        scale = np.abs(xa[:, :3] - sc.x[:, :3]).max()
        assert scale > 0  # the cloth moved
        # the same kernels on the same data (the batched PCG is bit-identical in and out of the mix, see
        # above); only float atomics (material and contact gradient / diagonal accumulation) add in another
        # order -- the contact pair list is ordered differently in a mix -- and 8 steps of contact amplify
        # that rounding (measured up to 2.8e-4 of the motion on a 900-vertex drape).  Stated tolerance: 1e-3
        # of the motion, or 3x the spread of two runs alone.
        spread = np.abs(xb[:, :3] - xa[:, :3]).max()
        dev = np.abs(xm[:, :3] - xa[:, :3]).max()
        print(f"\nscene {k}: in-mix deviation {dev / scale:.2e}, alone-vs-alone {spread / scale:.2e} of the motion")
        assert dev <= max(3.0 * spread, 1e-3 * scale) + 1e-7
        assert O.min_distance(sc, xm) > 0.0


def test_batched_newton_agrees_with_single_scene_solver():
    from luisacomputesimulator_b200.newton import NewtonSolver
    scs = _drapes()[:2]
    mix = NewtonBatch(scs)
    singles = [NewtonSolver(sc) for sc in scs]
    for _ in range(5):
        mix.step()
        for s in singles:
            s.step()
    for k, sc in enumerate(scs):
        xm, xs = mix.positions(k), singles[k].positions()
        scale = np.abs(xs[:, :3] - sc.x[:, :3]).max()
        np.testing.assert_allclose(xm[:, :3], xs[:, :3], rtol=0, atol=5e-3 * scale + 1e-7)


def _static_counts(sc, x):
    tf = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    te = O.lbvh_build(O.TREE_EDGE, x, sc.edges, sc.num_verts)
    O.lbvh_refit(tf, x, x, sc.faces, sc.offset)
    O.lbvh_refit(te, x, x, sc.edges, sc.offset)
    return O.lbvh_query_vf(tf, x, x, sc.d_hat, sc.offset)[1], O.lbvh_query_ee(te, x, x, sc.edges, sc.d_hat, sc.offset)[1]


def test_batch_with_a_body_filters_soft_scenes_and_traverses_the_rigid_one():
    """A batch holding an affine body: from the second Newton iteration of a step on, the soft scene's DCD lists
    come from filtering the previous CCD lists and the rigid scene's from a traversal of its trees.  The last
    iteration's candidate counts, summed over the scenes, equal the oracle's static queries at the positions that
    iteration started from."""
    import ctypes as C
    scs = [S.random_cloth_scene(900, 2), S.cloth_box_scene(600, 5)]
    batch = NewtonBatch(scs, nonlinear_iters=3)
    V = sum(sc.num_verts for sc in scs)
    offs = np.cumsum([0] + [sc.num_verts for sc in scs])
    checked = 0
    for _ in range(4):
        st = batch.step()
        assert st.status == 0
        if st.newton_iters < 2:
            continue
        x_iter = np.zeros((V, 4), np.float32)
        batch.lib.lcs_newton_last_iterate(batch.h, x_iter.ctypes.data_as(C.c_void_p), None, None)
        vf = ee = 0
        for k, sc in enumerate(scs):
            a, b = _static_counts(sc, x_iter[offs[k]:offs[k + 1]].copy())
            vf, ee = vf + a, ee + b
        assert (st.vf_candidates, st.ee_candidates) == (vf, ee)
        checked += 1
    assert checked >= 2
    for k, sc in enumerate(scs):
        assert O.min_distance(sc, batch.positions(k)) > 0.0
