"""Narrow-phase parity: CCD (bit-exact per-pair TOI, never above the oracle), DCD contact pairs
(identical sets, barrier stiffness within 1e-5 relative), gradient/diagonal assembly, the
off-diagonal BSR (bit-exact) and the contact energy."""
import numpy as np
import pytest
import torch

from luisacomputesimulator_b200.collision import NarrowPhasesDetector
from oracle import oracle as O
from tests import scenarios as SC
from tests.gpu_util import SceneOnDevice, counts, dev, host

pytestmark = pytest.mark.gpu


def _candidates(sc, x0, x1):
    tf = O.lbvh_build(O.TREE_FACE, x0, sc.faces, sc.num_verts)
    O.lbvh_refit(tf, x0, x1, sc.faces, sc.offset)
    vf, _ = O.lbvh_query_vf(tf, x0, x1, sc.d_hat, sc.offset)
    te = O.lbvh_build(O.TREE_EDGE, x0, sc.edges, sc.num_verts)
    O.lbvh_refit(te, x0, x1, sc.edges, sc.offset)
    ee, _ = O.lbvh_query_ee(te, x0, x1, sc.edges, sc.d_hat, sc.offset)
    return vf, ee


def _load(det, vf, ee):
    det.cap_vf = max(det.cap_vf, len(vf) + 1)
    det.cap_ee = max(det.cap_ee, len(ee) + 1)
    det._alloc()
    det.broad_phase_list_vf[: len(vf)] = dev(vf.astype(np.uint32))
    det.broad_phase_list_ee[: len(ee)] = dev(ee.astype(np.uint32))
    det.counts.zero_()
    det.counts[0] = len(vf)
    det.counts[1] = len(ee)


def _scenes():
    sc, x = SC.cloth_touching_sphere(gap=2e-3)
    x1 = x.copy()
    x1[: 64 * 64, 1] -= 6e-3  # the cloth moves through the sphere top
    yield "cloth_sphere", sc, x, x1
    sc, x = SC.folded_cloth(n=40, gap=3e-3)
    yield "folded", sc, x, SC.random_motion(x, 1.5e-3, seed=5)


SCENES = {name: (sc, x0, x1) for name, sc, x0, x1 in _scenes()}


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("fp64_final", [False, True])
def test_ccd_toi_bit_exact(name, fp64_final):
    sc, x0, x1 = SCENES[name]
    vf, ee = _candidates(sc, x0, x1)
    D = SceneOnDevice(sc)
    det = NarrowPhasesDetector(sc.num_verts, sc.edges.shape[0])
    _load(det, vf, ee)
    tvf = torch.zeros(det.cap_vf, dtype=torch.float32, device="cuda")
    tee = torch.zeros(det.cap_ee, dtype=torch.float32, device="cuda")
    det.reset_toi()
    det.vf_ccd_query(dev(x0), dev(x1), D.faces, D.body, D.offset, tvf, fp64_final)
    det.ee_ccd_query(dev(x0), dev(x1), D.edges, D.body, D.offset, tee, fp64_final)
    torch.cuda.synchronize()
    g_vf, o_vf = O.ccd_vf(vf, x0, x1, sc.faces, sc.body, sc.offset, fp64_final=fp64_final)
    g_ee, o_ee = O.ccd_ee(ee, x0, x1, sc.edges, sc.body, sc.offset, fp64_final=fp64_final)
    np.testing.assert_array_equal(host(tvf)[: len(vf)], o_vf)
    np.testing.assert_array_equal(host(tee)[: len(ee)], o_ee)
    g = float(host(det.toi)[0])
    assert g == min(g_vf, g_ee)
    assert g < 1.0  # the scenes do produce a step bound


def test_ccd_fp64_form_never_exceeds_fp32():
    sc, x0, x1 = SCENES["cloth_sphere"]
    vf, ee = _candidates(sc, x0, x1)
    _, a = O.ccd_vf(vf, x0, x1, sc.faces, sc.body, sc.offset, fp64_final=False)
    _, b = O.ccd_vf(vf, x0, x1, sc.faces, sc.body, sc.offset, fp64_final=True)
    assert np.all(b <= a)


def _dcd(name):
    sc, x0, _ = SCENES[name]
    if name == "cloth_sphere":
        sc, x0 = SC.cloth_touching_sphere(gap=4e-4)
    else:
        sc, x0 = SC.folded_cloth(n=40, gap=4e-4)
    vf, ee = _candidates(sc, x0, x0)
    D = SceneOnDevice(sc)
    det = NarrowPhasesDetector(sc.num_verts, sc.edges.shape[0])
    _load(det, vf, ee)
    xd = dev(x0)
    for attempt in range(2):  # resize-and-retry on overflow, as device_update_contact_list does
        det.reset_narrowphase_count()
        det.vf_dcd_query_repulsion(xd, D.faces, D.body, D.vert_area, D.face_area, D.d_hat, D.offset, sc.kappa)
        det.ee_dcd_query_repulsion(xd, D.edges, D.body, D.edge_area, D.d_hat, D.offset, sc.kappa)
        if not det.resize_buffers():
            break
        assert attempt == 0
    n = int(counts(det.counts)[2])
    assert n <= det.cap_pairs
    got = host(det.narrow_phase_list).view(O.PAIR_DTYPE).reshape(-1)[:n]
    want = np.concatenate([O.dcd_vf(vf, x0, sc.faces, sc.body, sc.vert_area, sc.face_area, sc.d_hat, sc.offset,
                                    sc.kappa),
                           O.dcd_ee(ee, x0, sc.edges, sc.body, sc.edge_area, sc.d_hat, sc.offset, sc.kappa)])
    return sc, x0, det, got, want


def _sort_pairs(p):
    k = p["idx"].astype(np.int64)
    order = np.lexsort((k[:, 3], k[:, 2], k[:, 1], k[:, 0]))
    return p[order]


@pytest.mark.parametrize("name", list(SCENES))
def test_dcd_pair_sets(name):
    sc, x0, det, got, want = _dcd(name)
    assert len(want) > 0 and len(got) == len(want)
    g, w = _sort_pairs(got), _sort_pairs(want)
    np.testing.assert_array_equal(g["idx"], w["idx"])
    np.testing.assert_array_equal(g["vec1"][:, :3], w["vec1"][:, :3])  # normal: bitwise
    np.testing.assert_array_equal(g["vec2"][:, 2:], w["vec2"][:, 2:])  # barycentrics: bitwise
    np.testing.assert_array_equal(g["vec1"][:, 3], w["vec1"][:, 3])  # kappa * area
    np.testing.assert_allclose(g["vec2"][:, :2], w["vec2"][:, :2], rtol=1e-5)  # k1, k2 (logf)


@pytest.mark.parametrize("name", list(SCENES))
def test_contact_assembly(name):
    sc, x0, det, got, want = _dcd(name)
    n = sc.num_verts
    # gradient + diagonal (atomics: order-free sums within FP32 tolerance)
    b = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    diag = torch.zeros((n, 3, 4), dtype=torch.float32, device="cuda")
    det.device_perPair_evaluate_gradient_hessian(b, diag)
    ob, od = O.contact_grad_diag(got, n)
    torch.cuda.synchronize()
    scale_b = np.abs(ob).max()
    scale_d = np.abs(od).max()
    np.testing.assert_allclose(host(b), ob, rtol=1e-5, atol=1e-6 * scale_b)
    np.testing.assert_allclose(host(diag), od, rtol=1e-5, atol=1e-6 * scale_d)
    # off-diagonal blocks: deterministic segmented sum, bitwise
    det.device_assemble_contact_triplet()
    rp, col, val = O.contact_offdiag_bsr(got, n)
    g_rp, g_col, g_val = det.assembler.export(n, 12 * len(got))
    assert g_col.shape[0] == len(col)
    np.testing.assert_array_equal(host(g_rp, np.uint32), rp)
    np.testing.assert_array_equal(host(g_col, np.uint32), col)
    np.testing.assert_array_equal(host(g_val), val)
    # energy
    det.reset_energy()
    det.compute_contact_energy(dev(x0), dev(sc.d_hat), dev(sc.offset))
    e = float(host(det.energy)[0])
    oe = O.contact_energy(got, x0, sc.d_hat, sc.offset, fp64=True)
    assert e == pytest.approx(oe, rel=1e-5)


@pytest.mark.parametrize("name", list(SCENES))
def test_ccd_fp64_form_matches_fp64_oracle(name):
    """The precision form's step bound: the ACCD iteration in FP64, bit-exact against the all-FP64
    oracle after rounding toward zero, so no per-pair TOI exceeds the FP64 value."""
    sc, x0, x1 = SCENES[name]
    vf, ee = _candidates(sc, x0, x1)
    D = SceneOnDevice(sc)
    det = NarrowPhasesDetector(sc.num_verts, sc.edges.shape[0])
    _load(det, vf, ee)
    tvf = torch.zeros(det.cap_vf, dtype=torch.float32, device="cuda")
    tee = torch.zeros(det.cap_ee, dtype=torch.float32, device="cuda")
    det.reset_toi()
    det.vf_ccd_query(dev(x0), dev(x1), D.faces, D.body, D.offset, tvf, fp64=True)
    det.ee_ccd_query(dev(x0), dev(x1), D.edges, D.body, D.offset, tee, fp64=True)
    torch.cuda.synchronize()
    for got, p, el, is_ee in ((host(tvf)[: len(vf)], vf, sc.faces, 0), (host(tee)[: len(ee)], ee, sc.edges, 1)):
        ref = O.ccd_f64(is_ee, p, x0, x1, el, sc.body, sc.offset)
        want = ref.astype(np.float32)
        want = np.where(want.astype(np.float64) > ref, np.nextafter(want, np.float32(0)), want)
        np.testing.assert_array_equal(got, want)
        assert np.all(got.astype(np.float64) <= ref)
        # and the FP32 form stays within 1e-6 relative of the FP64 iteration on these scenes
        _, t32 = (O.ccd_ee if is_ee else O.ccd_vf)(p, x0, x1, el, sc.body, sc.offset)
        m = ref < 1.25
        assert np.all(np.abs(t32[m] - ref[m]) <= 1e-6 * ref[m])
