"""Cloth energies on the GPU (lcs_eval_springs / lcs_eval_stretch_faces / lcs_eval_bending /
lcs_material_energy) against the oracle on the same inputs, through the C ABI.

Bars: springs and BW98 stretch bit-exact (same operation order, IEEE sqrt and division on both
sides); dihedral bending within 2e-6 of the largest magnitude (acosf differs between CUDA and
glibc by an ulp or so, which moves theta and everything scaled by it); energies (FP64 sums of FP32
terms, summation order differs) within 1e-5 relative."""
import ctypes as C

import numpy as np
import pytest
import torch

from luisacomputesimulator_b200 import _capi as A
from luisacomputesimulator_b200 import scenes as S
from oracle import oracle as O
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _deformed(sc, seed, amp):
    rng = np.random.default_rng(seed)
    x = sc.x.copy()
    x[:, :3] += rng.normal(0, amp, (sc.num_verts, 3)).astype(np.float32)
    return x


@pytest.fixture(scope="module")
def lib():
    return A.load()


@pytest.mark.parametrize("amp", [0.0, 1e-3, 5e-3])
def test_stretch_faces_bit_exact(lib, amp):
    sc = S.twisted_tube(40, 30)
    x = _deformed(sc, 0, amp)
    n = sc.stretch_faces.shape[0]
    ml = np.tile(np.float32([sc.stretch_mu, sc.stretch_lambda]), (n, 1))
    g_ref, h_ref = O.eval_stretch_faces(x, sc.stretch_faces, sc.stretch_dm_inv, sc.stretch_area, ml)
    g = torch.zeros((n, 3, 4), dtype=torch.float32, device="cuda")
    h = torch.zeros((n, 9, 3, 4), dtype=torch.float32, device="cuda")
    xs, fs, dm, ar, mlt = dev(x), dev(sc.stretch_faces), dev(sc.stretch_dm_inv), dev(sc.stretch_area), dev(ml)
    A.check(lib.lcs_eval_stretch_faces(_ptr(xs), _ptr(fs), _ptr(dm), _ptr(ar), _ptr(mlt), n, _ptr(g), _ptr(h), None),
            "lcs_eval_stretch_faces")
    torch.cuda.synchronize()
    assert np.array_equal(host(g), g_ref)
    assert np.array_equal(host(h), h_ref)


def test_springs_bit_exact(lib):
    sc = S.cloth_on_sphere(n=24)
    x = _deformed(sc, 1, 2e-3)
    n = sc.edges.shape[0]
    k = np.full(n, sc.spring_k, np.float32)
    g_ref, h_ref = O.eval_springs(x, sc.edges, sc.rest_len, k)
    g = torch.zeros((n, 2, 4), dtype=torch.float32, device="cuda")
    h = torch.zeros((n, 4, 3, 4), dtype=torch.float32, device="cuda")
    xs, es, rl, kk = dev(x), dev(sc.edges), dev(sc.rest_len), dev(k)
    A.check(lib.lcs_eval_springs(_ptr(xs), _ptr(es), _ptr(rl), _ptr(kk), n, _ptr(g), _ptr(h), None),
            "lcs_eval_springs")
    torch.cuda.synchronize()
    assert np.array_equal(host(g), g_ref)
    assert np.array_equal(host(h), h_ref)


@pytest.mark.parametrize("amp", [0.0, 2e-3])
def test_bending_matches_oracle(lib, amp):
    sc = S.twisted_tube(40, 30)
    x = _deformed(sc, 2, amp)
    n = sc.bending.shape[0]
    k = np.full(n, sc.bending_k, np.float32)
    g_ref, h_ref = O.eval_bending(x, sc.bending, sc.bending_rest_angle, sc.bending_hbar, k, sc.bending_scaling)
    g = torch.zeros((n, 4, 4), dtype=torch.float32, device="cuda")
    h = torch.zeros((n, 16, 3, 4), dtype=torch.float32, device="cuda")
    xs, st, ra, hb, kk = dev(x), dev(sc.bending), dev(sc.bending_rest_angle), dev(sc.bending_hbar), dev(k)
    A.check(lib.lcs_eval_bending(_ptr(xs), _ptr(st), _ptr(ra), _ptr(hb), _ptr(kk), float(sc.bending_scaling), n,
                                 _ptr(g), _ptr(h), None), "lcs_eval_bending")
    torch.cuda.synchronize()
    G, H = host(g), host(h)
    # the gradient is k (theta - rest) dtheta/dx: an acosf difference of d radians moves it by d k |dtheta/dx|,
    # and k |dtheta/dx_i| = sqrt(k trace(H_ii)); the bar is 1e-6 rad on top of 2e-6 relative
    stiff = (k * np.float32(sc.bending_scaling) * sc.bending_hbar).astype(np.float64)
    tr = np.einsum("sicc->si", h_ref[:, :4, :, :3].astype(np.float64))
    kg = np.sqrt(stiff[:, None] * tr).max()
    np.testing.assert_allclose(G, g_ref, rtol=0, atol=2e-6 * np.abs(g_ref).max() + 1e-6 * kg)
    np.testing.assert_allclose(H, h_ref, rtol=0, atol=2e-6 * np.abs(h_ref).max())
    exact = float(np.mean(H == h_ref))
    print(f"\nbending Hessian blocks bit-identical: {100 * exact:.1f} %")


def _cloth_elements(sc, x, xt):
    """lcs_cloth_elements of a scene's BW98 stretch faces and dihedral stencils (device copies in `keep`)."""
    Fs, B = sc.stretch_faces.shape[0], sc.bending.shape[0]
    keep = dict(x=dev(x), xt=dev(xt), mass=dev(sc.mass), fixed=dev(sc.pinned), f=dev(sc.stretch_faces),
                dm=dev(sc.stretch_dm_inv), ar=dev(sc.stretch_area),
                ml=dev(np.tile(np.float32([sc.stretch_mu, sc.stretch_lambda]), (Fs, 1))), st=dev(sc.bending),
                ra=dev(sc.bending_rest_angle), hb=dev(sc.bending_hbar), kb=dev(np.full(B, sc.bending_k, np.float32)))
    m = A.ClothElements()
    m.n_verts, m.n_springs, m.n_stretch_faces, m.n_bending = sc.num_verts, 0, Fs, B
    m.mass, m.is_fixed = _ptr(keep["mass"]), _ptr(keep["fixed"])
    m.stretch_faces, m.stretch_dm_inv, m.stretch_area = _ptr(keep["f"]), _ptr(keep["dm"]), _ptr(keep["ar"])
    m.stretch_mu_lambda = _ptr(keep["ml"])
    m.bending_edges, m.bending_rest_angle, m.bending_hbar = _ptr(keep["st"]), _ptr(keep["ra"]), _ptr(keep["hb"])
    m.bending_stiffness, m.bending_scaling = _ptr(keep["kb"]), sc.bending_scaling
    return m, keep


def test_material_energy_fp64(lib):
    sc = S.cloth_on_sphere(n=24)
    x = _deformed(sc, 3, 2e-3)
    xt = sc.x.copy()
    want = O.material_energy(sc, x, xt, sc.dt)
    m, keep = _cloth_elements(sc, x, xt)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    A.check(lib.lcs_material_energy(C.byref(m), _ptr(keep["x"]), _ptr(keep["xt"]), sc.dt, sc.dirichlet, _ptr(out),
                                    None), "lcs_material_energy")
    torch.cuda.synchronize()
    got = host(out)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-12)
