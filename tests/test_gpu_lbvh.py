"""LBVH parity: the CUDA build / refit / traversal against the oracle, bit for bit.

Sizes: config 1 (6,658 verts), a folded cloth (self contact), and config 2's 88,800-vertex
tube at full size (177,000-face and 265,800-edge trees)."""
import numpy as np
import pytest
import torch

from luisacomputesimulator_b200 import _capi as A
from luisacomputesimulator_b200.collision import LBVH
from oracle import oracle as O
from tests import scenarios as SC
from tests.gpu_util import SceneOnDevice, counts, dev, host

pytestmark = pytest.mark.gpu

KINDS = {"face": (O.TREE_FACE, "faces"), "edge": (O.TREE_EDGE, "edges")}


def _scene(name):
    if name == "cloth_sphere":
        return SC.cloth_touching_sphere(gap=5e-4)
    if name == "folded":
        return SC.folded_cloth(n=48, gap=4e-4)
    if name == "tube":
        return SC.twisted_tube_state(angle=1.2)
    if name == "tube_state":  # the benchmarked state: 56 steps of the run from rest
        sc, x, _, _ = SC.tube_state()
        return sc, x
    raise KeyError(name)


def _build_both(sc, x, kind_name):
    kind, attr = KINDS[kind_name]
    elems = getattr(sc, attr)
    t_o = O.lbvh_build(kind, x, elems, sc.num_verts)
    bvh = LBVH(kind, elems.shape[0])
    xd, ed = dev(x), dev(elems)
    if kind == O.TREE_FACE:
        bvh.reduce_face_tree_aabb(xd, ed)
    else:
        bvh.reduce_edge_tree_aabb(xd, ed)
    bvh.construct_tree()
    return t_o, bvh, xd, ed


@pytest.mark.parametrize("scene", ["cloth_sphere", "folded", "tube"])
@pytest.mark.parametrize("kind_name", ["face", "edge"])
def test_topology_bit_exact(scene, kind_name):
    sc, x = _scene(scene)
    t_o, bvh, _, _ = _build_both(sc, x, kind_name)
    assert bvh.check_health()
    e = bvh.export()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(e["global_aabb"]), np.concatenate([t_o.gmin, t_o.gmax]))
    np.testing.assert_array_equal(host(e["morton"], np.uint64), t_o.morton)
    np.testing.assert_array_equal(host(e["morton_sorted"], np.uint64), t_o.morton_sorted)
    np.testing.assert_array_equal(host(e["sorted_get_original"], np.uint32), t_o.sorted_get_original)
    np.testing.assert_array_equal(host(e["parent"], np.uint32), t_o.parent)
    np.testing.assert_array_equal(host(e["children"], np.uint32), t_o.children)
    np.testing.assert_array_equal(host(e["object_idx"], np.uint32), t_o.object_idx)


def _refit_both(kind, x, x1, elems, off):
    t_o = O.lbvh_build(kind, x, elems, x.shape[0])
    bvh = LBVH(kind, elems.shape[0])
    xd, ed = dev(x), dev(elems)
    if kind == O.TREE_FACE:
        bvh.reduce_face_tree_aabb(xd, ed)
    else:
        bvh.reduce_edge_tree_aabb(xd, ed)
    bvh.construct_tree()
    O.lbvh_refit(t_o, x, x1, elems, off)
    bvh.update_and_refit(dev(off), xd, dev(x1), ed)
    e = bvh.export()
    torch.cuda.synchronize()
    return t_o, host(e["node_aabb"])


@pytest.mark.parametrize("m", [2, 3, 40, 511, 512, 513, 1025, 1600])
def test_refit_bit_exact_across_chunk_sizes(m):
    """Trees of one, two and several 512-leaf refit chunks (the refit computes each inner box from its
    sorted leaf range, in one chunk or across chunks) against the oracle's bottom-up walk."""
    sc, x = _scene("folded")
    faces = np.ascontiguousarray(sc.faces[:m])
    x1 = SC.random_motion(x, 1e-3, seed=m)
    t_o, got = _refit_both(O.TREE_FACE, x, x1, faces, sc.offset + np.float32(1e-4))
    np.testing.assert_array_equal(got[:, 0:3], t_o.node_aabb[:, 0:3])
    np.testing.assert_array_equal(got[:, 4:7], t_o.node_aabb[:, 4:7])


def test_refit_signed_zero_ties_bit_exact():
    """Leaf boxes whose extremes tie at +0 and -0 (zero thickness, coordinates of both signs of zero): the
    reference's union `a < b ? a : b` keeps the later of two equal values, so the node boxes' zero signs
    depend on the order of the unions; compared as bit patterns."""
    rng = np.random.default_rng(3)
    g = 48
    ii, jj = np.meshgrid(np.arange(g), np.arange(g), indexing="ij")
    x = np.zeros((g * g, 4), np.float32)
    x[:, 0] = np.where(rng.random(g * g) < 0.5, np.float32(0.0), np.float32(-0.0))
    x[:, 1] = (ii.ravel() * 0.01).astype(np.float32)
    x[:, 2] = np.where(rng.random(g * g) < 0.5, np.float32(0.0), np.float32(-0.0))
    x[(jj.ravel() % 7) == 3, 2] = np.float32(0.01) * (jj.ravel()[(jj.ravel() % 7) == 3]).astype(np.float32)
    idx = (ii * g + jj)
    edges = np.concatenate([np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], 1),
                            np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], 1)]).astype(np.uint32)
    off = np.zeros(g * g, np.float32)
    t_o, got = _refit_both(O.TREE_EDGE, x, x.copy(), edges, off)
    assert (np.signbit(t_o.node_aabb[:, 0:3]).any() and (~np.signbit(t_o.node_aabb[:, 0:3])).any())
    np.testing.assert_array_equal(got[:, 0:3].view(np.uint32), t_o.node_aabb[:, 0:3].view(np.uint32))
    np.testing.assert_array_equal(got[:, 4:7].view(np.uint32), t_o.node_aabb[:, 4:7].view(np.uint32))


@pytest.mark.parametrize("scene", ["cloth_sphere", "folded", "tube"])
@pytest.mark.parametrize("kind_name", ["face", "edge"])
@pytest.mark.parametrize("fused", [False, True])
def test_refit_bit_exact(scene, kind_name, fused):
    sc, x = _scene(scene)
    t_o, bvh, xd, ed = _build_both(sc, x, kind_name)
    x1 = SC.random_motion(x, 1e-3, seed=7)
    x1d = dev(x1)
    off = dev(sc.offset + np.float32(1e-4))
    O.lbvh_refit(t_o, x, x1, getattr(sc, KINDS[kind_name][1]), sc.offset + np.float32(1e-4))
    for _ in range(2):  # twice: a refit over its own previous output
        if fused:
            bvh.update_and_refit(off, xd, x1d, ed)
        else:
            bvh.update_leaves(off, xd, x1d, ed)
            bvh.refit()
    e = bvh.export()
    torch.cuda.synchronize()
    got = host(e["node_aabb"])
    np.testing.assert_array_equal(got[:, 0:3], t_o.node_aabb[:, 0:3])
    np.testing.assert_array_equal(got[:, 4:7], t_o.node_aabb[:, 4:7])


@pytest.mark.parametrize("scene", ["cloth_sphere", "folded", "tube", "tube_state"])
@pytest.mark.parametrize("swept", [False, True])
def test_candidate_sets_bit_exact(scene, swept):
    sc, x = _scene(scene)
    x1 = SC.random_motion(x, 2e-3, seed=11) if swept else x
    D = SceneOnDevice(sc)
    xd, x1d = dev(x), dev(x1)
    for kind_name in ("face", "edge"):
        t_o, bvh, _, ed = _build_both(sc, x, kind_name)
        elems = getattr(sc, KINDS[kind_name][1])
        O.lbvh_refit(t_o, x, x1, elems, sc.offset)
        bvh.update_and_refit(D.offset, xd, x1d, ed)
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        if kind_name == "face":
            want, n_want = O.lbvh_query_vf(t_o, x, x1, sc.d_hat, sc.offset)
            pairs = torch.zeros((n_want + 64, 2), dtype=torch.int32, device="cuda")
            bvh.broad_phase_query_from_verts(xd, x1d, cnt, pairs, D.d_hat, D.offset)
        else:
            want, n_want = O.lbvh_query_ee(t_o, x, x1, sc.edges, sc.d_hat, sc.offset)
            pairs = torch.zeros((n_want + 64, 2), dtype=torch.int32, device="cuda")
            bvh.broad_phase_query_from_edges(xd, x1d, D.edges, cnt, pairs, D.d_hat, D.offset)
        n = int(counts(cnt)[0])
        assert n == n_want
        got = host(pairs, np.uint32)[:n]
        np.testing.assert_array_equal(SC.sorted_pairs(got), SC.sorted_pairs(want))


def test_update_and_refit_before_construct_is_refused():
    """Leaf order, slots and refit tables come from the build: before it, update / refit / query / export
    are refused (LCS_ERR_INVALID) instead of reading tables that hold no indices; after it they run."""
    sc, x = _scene("folded")
    faces = np.ascontiguousarray(sc.faces[:700])
    edges = np.ascontiguousarray(sc.edges[:900])
    bvh = LBVH(O.TREE_FACE, faces.shape[0])
    ebvh = LBVH(O.TREE_EDGE, edges.shape[0])
    xd, fd, edd, off, dh = dev(x), dev(faces), dev(edges), dev(sc.offset), dev(sc.d_hat)
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.zeros((1024, 2), dtype=torch.int32, device="cuda")
    for call in (lambda: bvh.update_and_refit(off, xd, xd, fd), lambda: bvh.update_leaves(off, xd, xd, fd),
                 bvh.refit, bvh.export, lambda: bvh.broad_phase_query_from_verts(xd, xd, cnt, pairs, dh, off),
                 lambda: ebvh.broad_phase_query_from_edges(xd, xd, edd, cnt, pairs, dh, off),
                 lambda: ebvh.broad_phase_query_from_edges_sym(xd, xd, edd, cnt, pairs, float(sc.d_hat[0]))):
        with pytest.raises(A.LcsError, match="LCS_ERR_INVALID"):
            call()
    bvh.reduce_face_tree_aabb(xd, fd)
    bvh.construct_tree()
    bvh.update_and_refit(off, xd, xd, fd)
    bvh.broad_phase_query_from_verts(xd, xd, cnt, pairs, dh, off)
    torch.cuda.synchronize()
    assert bvh.check_health()


def test_query_overflow_counts_without_writing_past_capacity():
    sc, x = _scene("cloth_sphere")
    D = SceneOnDevice(sc)
    t_o, bvh, xd, ed = _build_both(sc, x, "edge")
    bvh.update_and_refit(D.offset, xd, xd, ed)
    O.lbvh_refit(t_o, x, x, sc.edges, sc.offset)
    want, n_want = O.lbvh_query_ee(t_o, x, x, sc.edges, sc.d_hat, sc.offset)
    cap = 1000
    guard = torch.full((cap + 16, 2), -7, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    bvh.broad_phase_query_from_edges(xd, xd, D.edges, cnt, guard[:cap], D.d_hat, D.offset)
    n = int(counts(cnt)[0])
    assert n == n_want and n > cap
    g = host(guard)
    assert np.all(g[cap:] == -7)  # nothing past capacity
    full = {tuple(p) for p in SC.sorted_pairs(want).tolist()}
    assert all(tuple(p) in full for p in g[:cap].astype(np.int64).tolist())


def test_single_leaf_tree_and_empty_queries():
    # one face: the reference's root is the leaf itself and both child reads hit it
    x = np.array([[0, 0, 0, 0], [1, 0, 0, 0], [0, 1, 0, 0], [0.2, 0.2, 0.0005, 0]], np.float32)
    faces = np.array([[0, 1, 2, 0]], np.uint32)
    t_o = O.lbvh_build(O.TREE_FACE, x, faces, 4)
    thick = np.zeros(4, np.float32)
    dhat = np.full(4, 1e-3, np.float32)
    O.lbvh_refit(t_o, x, x, faces, thick)
    want, n_want = O.lbvh_query_vf(t_o, x, x, dhat, thick)
    bvh = LBVH(O.TREE_FACE, 1)
    xd, fd = dev(x), dev(faces)
    bvh.reduce_face_tree_aabb(xd, fd)
    bvh.construct_tree()
    bvh.update_and_refit(dev(thick), xd, xd, fd)
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.zeros((16, 2), dtype=torch.int32, device="cuda")
    bvh.broad_phase_query_from_verts(xd, xd, cnt, pairs, dev(dhat), dev(thick))
    n = int(counts(cnt)[0])
    assert n == n_want
    np.testing.assert_array_equal(SC.sorted_pairs(host(pairs, np.uint32)[:n]), SC.sorted_pairs(want))


@pytest.mark.parametrize("scene", ["cloth_sphere", "folded"])
def test_filtered_swept_lists_equal_static_queries_on_the_sweep(scene):
    """The fused Newton loop takes its DCD candidates from the previous CCD lists: filtering the swept
    list (x0 -> x1) at any x = x0 + t (x1 - x0), 0 <= t <= 1, must give the static-box list at x."""
    import ctypes as C
    from luisacomputesimulator_b200 import _capi as A
    from luisacomputesimulator_b200.collision import ptr, stream
    sc, x0 = _scene(scene)
    x1 = SC.random_motion(x0, 2e-3, seed=3)
    xm = x0.copy()
    xm[:, :3] = x0[:, :3] + np.float32(0.37) * (x1[:, :3] - x0[:, :3])
    D = SceneOnDevice(sc)
    lib = A.load()
    for kind_name, is_ee in (("face", 0), ("edge", 1)):
        t_o, bvh, _, ed = _build_both(sc, x0, kind_name)
        elems = getattr(sc, KINDS[kind_name][1])
        bvh.update_and_refit(D.offset, dev(x0), dev(x1), ed)
        cap = 64 * max(sc.num_verts, elems.shape[0])
        swept = torch.zeros((cap, 2), dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        if is_ee:
            bvh.broad_phase_query_from_edges(dev(x0), dev(x1), D.edges, cnt, swept, D.d_hat, D.offset)
        else:
            bvh.broad_phase_query_from_verts(dev(x0), dev(x1), cnt, swept, D.d_hat, D.offset)
        assert int(counts(cnt)[0]) <= cap  # the whole swept list was written
        out = torch.zeros((cap, 2), dtype=torch.int32, device="cuda")
        ocnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        A.check(lib.lcs_candidates_filter(is_ee, ptr(swept), ptr(cnt), cap, ptr(dev(xm)), ptr(ed), ptr(D.d_hat),
                                          ptr(D.offset), ptr(out), cap, ptr(ocnt), stream()), "filter")
        O.lbvh_refit(t_o, xm, xm, elems, sc.offset)
        if is_ee:
            want, n_want = O.lbvh_query_ee(t_o, xm, xm, sc.edges, sc.d_hat, sc.offset)
        else:
            want, n_want = O.lbvh_query_vf(t_o, xm, xm, sc.d_hat, sc.offset)
        n = int(counts(ocnt)[0])
        assert n == n_want and n <= int(counts(cnt)[0])
        np.testing.assert_array_equal(SC.sorted_pairs(host(out, np.uint32)[:n]), SC.sorted_pairs(want))


@pytest.mark.parametrize("scene", ["cloth_sphere", "folded", "tube", "tube_state"])
@pytest.mark.parametrize("swept", [False, True])
def test_once_per_pair_ee_query_matches_the_reference_set(scene, swept):
    """lcs_bvh_query_ee_sym (each pair met once, from the lower Morton position) returns the oracle's
    EE set bit for bit on scenes with thickness 0 and one d_hat -- the Newton loop's configuration."""
    sc, x = _scene(scene)
    sc.offset = np.zeros_like(sc.offset)
    sc.d_hat = np.full_like(sc.d_hat, sc.d_hat[sc.edges[0, 0]])
    x1 = SC.random_motion(x, 2e-3, seed=13) if swept else x
    D = SceneOnDevice(sc)
    xd, x1d = dev(x), dev(x1)
    t_o, bvh, _, ed = _build_both(sc, x, "edge")
    O.lbvh_refit(t_o, x, x1, sc.edges, sc.offset)
    bvh.update_and_refit(D.offset, xd, x1d, ed)
    want, n_want = O.lbvh_query_ee(t_o, x, x1, sc.edges, sc.d_hat, sc.offset)
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.zeros((n_want + 64, 2), dtype=torch.int32, device="cuda")
    bvh.broad_phase_query_from_edges_sym(xd, x1d, D.edges, cnt, pairs, float(sc.d_hat[0]))
    n = int(counts(cnt)[0])
    assert n == n_want
    np.testing.assert_array_equal(SC.sorted_pairs(host(pairs, np.uint32)[:n]), SC.sorted_pairs(want))


def test_once_per_pair_ee_query_on_boxes_at_the_threshold():
    """A grid whose edge boxes sit at distance d_hat from each other on every axis (spacing = edge length
    + d_hat, scaled so the sums round): the strict test decides at the last ulp, from either side."""
    rng = np.random.default_rng(5)
    n = 40
    d = np.float32(1e-3)
    seg = []
    for i in range(n):
        for j in range(n):
            p = np.array([i * 3e-3, j * 3e-3, 0.0], np.float32)
            seg.append((p, p + np.array([2e-3, 0, 0], np.float32)))
            seg.append((p + np.array([0, 1e-3, 0], np.float32),
                        p + np.array([0, 1e-3, 0], np.float32) + np.float32(1e-3) * rng.normal(size=3).astype(np.float32)))
    x = np.zeros((2 * len(seg), 4), np.float32)
    for k, (a, b) in enumerate(seg):
        x[2 * k, :3], x[2 * k + 1, :3] = a, b
    edges = np.arange(2 * len(seg), dtype=np.uint32).reshape(-1, 2)
    V = x.shape[0]
    dh, off = np.full(V, d, np.float32), np.zeros(V, np.float32)
    t_o = O.lbvh_build(O.TREE_EDGE, x, edges, V)
    O.lbvh_refit(t_o, x, x, edges, off)
    want, n_want = O.lbvh_query_ee(t_o, x, x, edges, dh, off)
    bvh = LBVH(O.TREE_EDGE, edges.shape[0])
    xd, ed = dev(x), dev(edges)
    bvh.reduce_edge_tree_aabb(xd, ed)
    bvh.construct_tree()
    bvh.update_and_refit(dev(off), xd, xd, ed)
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.zeros((n_want + 64, 2), dtype=torch.int32, device="cuda")
    bvh.broad_phase_query_from_edges_sym(xd, xd, ed, cnt, pairs, float(d))
    m = int(counts(cnt)[0])
    assert m == n_want and n_want > 0
    np.testing.assert_array_equal(SC.sorted_pairs(host(pairs, np.uint32)[:m]), SC.sorted_pairs(want))


def _deep_tree(kind_name):
    x, el = SC.deep_tree_elements(kind_name)
    V = x.shape[0]
    kind = KINDS[kind_name][0]
    t_o = O.lbvh_build(kind, x, el, V)
    bvh = LBVH(kind, el.shape[0])
    xd, ed = dev(x), dev(el)
    if kind == O.TREE_FACE:
        bvh.reduce_face_tree_aabb(xd, ed)
    else:
        bvh.reduce_edge_tree_aabb(xd, ed)
    bvh.construct_tree()
    z = np.zeros(V, np.float32)
    O.lbvh_refit(t_o, x, x, el, z)
    bvh.update_and_refit(dev(z), xd, xd, ed)
    return x, el, t_o, bvh, xd, ed


def _brute_force_count(x, el, r, ee):
    """Size of the complete candidate set (strict box overlap, no early exit)."""
    m = 2 if ee else 3
    lo, hi = x[el[:, :m], :3].min(1), x[el[:, :m], :3].max(1)
    if ee:  # edge i's query box: its box widened by r of its first vertex; pairs i < j
        rq = r[el[:, 0]][:, None]
        qlo, qhi = lo - rq, hi + rq
    else:  # vertex v's query box: the point widened by r[v]
        qlo, qhi = x[:, :3] - r[:, None], x[:, :3] + r[:, None]
    ov = (lo[None] < qhi[:, None]).all(2) & (hi[None] > qlo[:, None]).all(2)
    if ee:
        i, j = np.nonzero(ov)
        return int((i < j).sum())
    return int(ov.sum())


@pytest.mark.parametrize("kind_name", ["face", "edge"])
def test_deep_tree_traversal_ends_early_like_the_reference(kind_name):
    """A tree with inner nodes at depth >= 32, where the reference's 32-entry stack fills: every query whose
    walk meets a full stack ends there, keeping only the pairs found before (lbvh.cpp:293-360).  Per-vertex
    query radii mix queries that end early with queries that finish.  The GPU sets equal the oracle's, which
    are smaller than the complete sets; the early exit is reported."""
    x, el, t_o, bvh, xd, ed = _deep_tree(kind_name)
    V = x.shape[0]
    r = np.random.default_rng(7).uniform(200.0, 800.0, V).astype(np.float32)
    z = np.zeros(V, np.float32)
    ee = kind_name == "edge"
    if ee:
        want, n_want = O.lbvh_query_ee(t_o, x, x, el, r, z)
    else:
        want, n_want = O.lbvh_query_vf(t_o, x, x, r, z)
    assert 0 < n_want < _brute_force_count(x, el, r, ee)  # the reference's early exit removed pairs
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    pairs = torch.zeros((n_want + 64, 2), dtype=torch.int32, device="cuda")
    if ee:
        bvh.broad_phase_query_from_edges(xd, xd, ed, cnt, pairs, dev(r), dev(z))
    else:
        bvh.broad_phase_query_from_verts(xd, xd, cnt, pairs, dev(r), dev(z))
    n = int(counts(cnt)[0])
    assert n == n_want
    np.testing.assert_array_equal(SC.sorted_pairs(host(pairs, np.uint32)[:n]), SC.sorted_pairs(want))


def test_deep_tree_once_per_pair_query_falls_back_to_the_reference_walk():
    """The once-per-pair EE form relies on the set being symmetric, which the reference's early exit breaks:
    on a deep tree lcs_bvh_query_ee_sym runs the reference's full EE walk and returns its set."""
    x, el, t_o, bvh, xd, ed = _deep_tree("edge")
    V = x.shape[0]
    z = np.zeros(V, np.float32)
    for rad in (300.0, 520.0, 600.0):
        r = np.full(V, rad, np.float32)
        want, n_want = O.lbvh_query_ee(t_o, x, x, el, r, z)
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        pairs = torch.zeros((max(n_want, 1) + 64, 2), dtype=torch.int32, device="cuda")
        bvh.broad_phase_query_from_edges_sym(xd, xd, ed, cnt, pairs, rad)
        n = int(counts(cnt)[0])
        assert n == n_want, (rad, n, n_want)
        np.testing.assert_array_equal(SC.sorted_pairs(host(pairs, np.uint32)[:n]), SC.sorted_pairs(want))
