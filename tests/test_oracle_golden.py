"""Pins the CPU oracle to the reference's own known answers (tests/golden/) and checks its
internal invariants.  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import scenarios as SC

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.json")))


def test_morton_codes_match_reference_unit_test():
    g = GOLD["lbvh_unit"]
    m32, m64 = O.morton_unit(g["leaves"])
    assert m32.tolist() == g["morton32"]
    assert m64.astype(np.uint64).tolist() == g["morton64"]


def test_karras_topology_matches_reference_comments():
    g = GOLD["lbvh_unit"]
    _, m64 = O.morton_unit(g["leaves"])
    t = O.build_inner(m64)
    assert t["healthy"] == 1
    assert t["ranges"].tolist() == g["ranges"]
    assert t["splits"].tolist() == g["splits"]
    assert t["children"][:7].tolist() == g["children"]
    assert t["parent"][1:].tolist() == g["parents_nonroot"]
    assert int(t["parent"][0]) == 0xFFFFFFFF


@pytest.mark.parametrize("depth", GOLD["refit_complete_tree"]["depths"])
def test_refit_complete_tree_root(depth):
    # UnitTest/test_lbvh_refit.cpp:253-349: leaf i has box [i, i+1]^3, root must be [0, 2^depth]^3
    n = 1 << depth
    ni = n - 1
    parent = np.zeros(2 * n - 1, np.uint32)
    children = np.zeros((2 * n - 1, 2), np.uint32)
    for i in range(ni):
        children[i] = (2 * i + 1, 2 * i + 2)
    for k in range(1, 2 * n - 1):
        parent[k] = (k - 1) // 2
    parent[0] = 0xFFFFFFFF
    aabb = np.zeros((2 * n - 1, 8), np.float32)
    for i in range(n):
        aabb[ni + i] = [i, i, i, 0, i + 1, i + 1, i + 1, 1]
    L = O.lib()
    ok = L.orc_lbvh_refit(n, O._p(parent), O._p(children), O._p(aabb))
    assert ok == 1
    assert aabb[0, :3].tolist() == [0.0, 0.0, 0.0]
    assert aabb[0, 4:7].tolist() == [float(n)] * 3


def test_vf_ccd_known_answer():
    g = GOLD["vf_ccd"]
    toi = O.point_triangle_ccd(g["t0_p"], g["t1_p"], g["t0_f0"], g["t0_f1"], g["t0_f2"], g["t1_f0"], g["t1_f1"],
                               g["t1_f2"], g["offset"])
    assert abs(toi - g["desire_toi"]) <= 1e-6 * g["desire_toi"]
    # the FP64-checked precision form never exceeds the FP32 bound
    toi64 = O.point_triangle_ccd(g["t0_p"], g["t1_p"], g["t0_f0"], g["t0_f1"], g["t0_f2"], g["t1_f0"], g["t1_f1"],
                                 g["t1_f2"], g["offset"], fp64_final=True)
    assert toi64 <= toi and toi64 > 0.99 * toi


def test_ee_ccd_case_runs_and_is_bounded():
    g = GOLD["ee_ccd"]
    args = [g[k] for k in ("ea_t0_p0", "ea_t0_p1", "eb_t0_p0", "eb_t0_p1", "ea_t1_p0", "ea_t1_p1", "eb_t1_p0",
                           "eb_t1_p1")]
    for th in (0.0, g["thickness"]):
        toi = O.edge_edge_ccd(*args, th)
        assert np.isfinite(toi) and toi <= 1.25


def test_barrier_derivatives_against_fp64():
    for d, dhat in [(1.9e-4, 1e-3), (5e-4, 1e-3), (9.9e-4, 1e-3), (1e-5, 3e-5)]:
        b, db, ddb = O.barrier(d, dhat)
        dd, hh = np.float64(d), np.float64(dhat)
        ref_b = -(dd - hh) ** 2 * np.log(dd / hh)
        ref_db = (hh - dd) * (2 * np.log(dd / hh) - hh / dd + 1)
        ref_ddb = (hh / dd + 2) * (hh / dd) - 2 * np.log(dd / hh) - 3
        assert b == pytest.approx(ref_b, rel=1e-4, abs=1e-12)
        assert db == pytest.approx(ref_db, rel=1e-4, abs=1e-9)
        assert ddb == pytest.approx(ref_ddb, rel=1e-4)


def test_lbvh_candidates_cover_brute_force():
    # every (vertex, face) pair whose boxes overlap strictly is reported exactly once
    sc, x = SC.folded_cloth(n=12, gap=4e-4)
    t = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    assert t.healthy
    O.lbvh_refit(t, x, x, sc.faces, sc.offset)
    pairs, cnt = O.lbvh_query_vf(t, x, x, sc.d_hat, sc.offset)
    got = SC.sorted_pairs(pairs)
    xv = x[:, :3]
    fmin = np.minimum(np.minimum(xv[sc.faces[:, 0]], xv[sc.faces[:, 1]]), xv[sc.faces[:, 2]])
    fmax = np.maximum(np.maximum(xv[sc.faces[:, 0]], xv[sc.faces[:, 1]]), xv[sc.faces[:, 2]])
    r = (sc.d_hat + sc.offset)[:, None]
    qmin, qmax = xv - r, xv + r
    ov = np.all(fmin[None, :, :] < qmax[:, None, :], -1) & np.all(fmax[None, :, :] > qmin[:, None, :], -1)
    want = SC.sorted_pairs(np.argwhere(ov))
    assert cnt == len(want)
    np.testing.assert_array_equal(got, want)


def test_dcd_pairs_are_within_dhat_and_assembly_is_symmetric():
    sc, x = SC.folded_cloth(n=16, gap=4e-4)
    t = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    O.lbvh_refit(t, x, x, sc.faces, sc.offset)
    cand, _ = O.lbvh_query_vf(t, x, x, sc.d_hat, sc.offset)
    pairs = O.dcd_vf(cand, x, sc.faces, sc.body, sc.vert_area, sc.face_area, sc.d_hat, sc.offset, sc.kappa)
    assert len(pairs) > 0
    assert np.all(pairs["vec2"][:, 1] > 0)  # k2 > 0 inside d_hat
    rp, col, val = O.contact_offdiag_bsr(pairs, sc.num_verts)
    # dense check: the off-diagonal contact Hessian is symmetric
    n = sc.num_verts
    M = {}
    for r in range(n):
        for k in range(rp[r], rp[r + 1]):
            M[(r, int(col[k]))] = val[k].reshape(3, 3).T  # column-major block
    for (r, c), blk in M.items():
        np.testing.assert_allclose(blk, M[(c, r)].T, rtol=1e-5, atol=1e-3)


def test_pcg_solves_spd_system():
    rng = np.random.default_rng(3)
    n = 60
    # SPD block system: diag blocks dominant, symmetric off-diagonal blocks on a ring
    diag = np.zeros((n, 3, 4), np.float32)
    for i in range(n):
        a = rng.normal(size=(3, 3))
        m = a @ a.T + 8 * np.eye(3)
        diag[i, :, :3] = m.T  # column-major columns
    rows, cols, vals = [], [], []
    for i in range(n):
        for j in ((i + 1) % n, (i - 1) % n):
            rows.append(i)
            cols.append(j)
            vals.append(-0.5 * np.eye(3))
    order = np.lexsort((cols, rows))
    rows, cols = np.asarray(rows)[order], np.asarray(cols)[order]
    vals = np.asarray(vals)[order]
    rp = np.zeros(n + 1, np.uint32)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    val9 = np.stack([v.T.reshape(9) for v in vals]).astype(np.float32)
    b = np.zeros((n, 4), np.float32)
    b[:, :3] = rng.normal(size=(n, 3))
    x, st = O.pcg(diag, (rp, cols.astype(np.uint32), val9), None, b, max_iter=200, rel_tol=1e-6, check_every=1,
                  fp64_dots=True)
    K = np.zeros((3 * n, 3 * n))
    for i in range(n):
        K[3 * i:3 * i + 3, 3 * i:3 * i + 3] = diag[i, :, :3].T
    for r, c, v in zip(rows, cols, vals):
        K[3 * r:3 * r + 3, 3 * c:3 * c + 3] += v
    ref = np.linalg.solve(K, b[:, :3].reshape(-1).astype(np.float64))
    assert st["status"] == 0 and st["rel_residual"] <= 1e-6
    np.testing.assert_allclose(x[:, :3].reshape(-1), ref, rtol=1e-4, atol=1e-5)


def test_fp64_ccd_oracle_close_to_fp32_and_known_answer():
    """The all-FP64 ACCD (error reference of the precision form) agrees with the FP32 iteration to
    about float precision and reproduces the point-triangle known answer."""
    import numpy as np
    from tests import scenarios as SC
    sc, x = SC.cloth_touching_sphere(gap=2e-3)
    x1 = x.copy()
    x1[: 64 * 64, 1] -= 6e-3
    tf = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    O.lbvh_refit(tf, x, x1, sc.faces, sc.offset)
    vf, _ = O.lbvh_query_vf(tf, x, x1, sc.d_hat, sc.offset)
    ref = O.ccd_f64(0, vf, x, x1, sc.faces, sc.body, sc.offset)
    _, t32 = O.ccd_vf(vf, x, x1, sc.faces, sc.body, sc.offset)
    m = ref < 1.25
    assert m.sum() > 50
    assert np.all(np.abs(t32[m] - ref[m]) <= 1e-6 * ref[m])
    g = GOLD["vf_ccd"]
    x0 = np.array([g["t0_p"], g["t0_f0"], g["t0_f1"], g["t0_f2"]], np.float32)
    x1 = np.array([g["t1_p"], g["t1_f0"], g["t1_f1"], g["t1_f2"]], np.float32)
    off = np.array([g["offset"] / 2] * 4, np.float32)
    toi = O.ccd_f64(0, np.array([[0, 0]], np.uint32), x0, x1, np.array([[1, 2, 3, 0]], np.uint32),
                    np.full(4, 0xFFFFFFFF, np.uint32), off)[0]
    assert abs(toi - g["desire_toi"]) <= 1e-6 * g["desire_toi"]
