"""The oracle's cloth energies (oracle/lcs_oracle_material.c) against float64 restatements of the
reference's matrix forms, on the CPU:

* BW98 stretch + shear: gradient = dF/dx^T dE/dF (convert_force) and Hessian = dF/dx^T H dF/dx
  (convert_hessian) with H the projected 6x6 Hessian of detail::stretch_hessian / shear_hessian
  (Solver/Energy/stretch_energy.h:156-321), written here as the reference writes it (the q0, T, lambda0
  construction on the flattened F); the gradient also against central differences of the energy
  (compute_energy, stretch_energy.h:508-520);
* dihedral bending: the angle of face_dihedral_angle and the gradient of face_dihedral_angle_grad
  (Solver/Energy/bending_energy.h:167-231) against central differences of the angle;
* the elastic energy sums (fn_calc_energy_*, Solver/SimulationSolver/solver_interface.cpp:505-728);
* the fused fill (orc_material_fill2) against the per-element outputs assembled in numpy.
"""
import numpy as np
import pytest

from luisacomputesimulator_b200 import scenes as S
from oracle import newton_cpu as N
from oracle import oracle as O


def _F(x0, x1, x2, dm):
    Dm = np.array([[dm[0], dm[2]], [dm[1], dm[3]]], np.float64)
    return np.stack([x1 - x0, x2 - x0], 1) @ Dm  # 3 x 2


def _energy64(x0, x1, x2, dm, mu, lam, area):
    F = _F(x0, x1, x2, dm)
    su, sv, i6 = np.linalg.norm(F[:, 0]), np.linalg.norm(F[:, 1]), F[:, 0] @ F[:, 1]
    return area * (0.5 * mu * ((su - 1) ** 2 + (sv - 1) ** 2) + 0.5 * lam * i6 ** 2)


def _reference_matrix_form(x0, x1, x2, dm, mu, lam, area):
    """stretch_energy.h in float64: flattened F = [Fu; Fv] (6), projected 6x6 Hessian, chain rule."""
    F = _F(x0, x1, x2, dm)
    Fu, Fv = F[:, 0], F[:, 1]
    su, sv = np.linalg.norm(Fu), np.linalg.norm(Fv)
    I6 = Fu @ Fv
    dedF = np.concatenate([mu * (su - 1) / su * Fu + lam * I6 * Fv, mu * (sv - 1) / sv * Fv + lam * I6 * Fu])
    H = np.zeros((6, 6))
    for blk, s, f in ((0, su, Fu), (1, sv, Fv)):  # stretch_hessian
        fn = f / s
        H[3 * blk:3 * blk + 3, 3 * blk:3 * blk + 3] = mu * (max(0.0, 1 - 1 / s) * np.eye(3) +
                                                           min(1 / s, 1.0) * np.outer(fn, fn))
    S6 = np.zeros((6, 6))  # shear_hessian
    S6[3:, :3] = S6[:3, 3:] = np.eye(3)
    g = np.concatenate([Fv, Fu])
    I2 = Fu @ Fu + Fv @ Fv
    lam0 = 0.5 * (I2 + np.sqrt(I2 * I2 + 12 * I6 * I6))
    q0 = I6 * S6 @ g + lam0 * g
    q0 /= np.linalg.norm(q0)
    T = 0.5 * (np.eye(6) + np.sign(I6) * S6)
    Tq = T @ q0
    H += lam * (abs(I6) * (T - np.outer(Tq, Tq) / (Tq @ Tq)) + lam0 * np.outer(q0, q0))
    J = np.zeros((6, 9))  # dF/dx (get_dFdx)
    d0, d1, d2, d3 = dm
    w = [(-(d0 + d1), -(d2 + d3)), (d0, d2), (d1, d3)]
    for a in range(3):
        for c in range(2):
            J[3 * c:3 * c + 3, 3 * a:3 * a + 3] = w[a][c] * np.eye(3)
    return area * J.T @ dedF, area * J.T @ H @ J


def _triangles(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        X = rng.normal(0, 0.01, (3, 3))
        dm = S._dm_inv(X, np.array([[0, 1, 2]]))[0].astype(np.float64)
        A = np.eye(3) + rng.normal(0, 0.3, (3, 3))  # stretch, compress and shear the rest shape
        x = (X @ A.T + rng.normal(0, 0.002, (3, 3))).astype(np.float32)
        area = 0.5 * np.linalg.norm(np.cross(X[1] - X[0], X[2] - X[0]))
        out.append((x, dm.astype(np.float32), float(np.float32(area))))
    return out


def _full9(K6):
    K = np.zeros((9, 9))
    for k, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
        blk = K6[k].reshape(3, 3).T  # column-major -> [row, col]
        K[3 * a:3 * a + 3, 3 * b:3 * b + 3] = blk
        K[3 * b:3 * b + 3, 3 * a:3 * a + 3] = blk.T
    return K


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_bw98_oracle_matches_reference_matrix_form(seed):
    mu, lam = S.lame()
    for x, dm, area in _triangles(40, seed):
        g, K6 = O.bw98_face(x[0], x[1], x[2], dm, mu, lam, area)
        x64, dm64 = x.astype(np.float64), dm.astype(np.float64)
        g_ref, K_ref = _reference_matrix_form(x64[0], x64[1], x64[2], dm64, mu, lam, area)
        scale_g = np.abs(g_ref).max() + 1e-12
        np.testing.assert_allclose(g.reshape(-1), g_ref, rtol=0, atol=2e-4 * scale_g)
        K = _full9(K6)
        np.testing.assert_allclose(K, K_ref, rtol=0, atol=2e-4 * np.abs(K_ref).max())
        assert np.linalg.eigvalsh(K_ref).min() >= -1e-9 * np.abs(K_ref).max()  # projected: PSD
        # the gradient is the derivative of compute_energy
        h = 1e-7
        fd = np.zeros(9)
        for i in range(9):
            xp, xm = x64.copy(), x64.copy()
            xp.reshape(-1)[i] += h
            xm.reshape(-1)[i] -= h
            fd[i] = (_energy64(*xp, dm64, mu, lam, area) - _energy64(*xm, dm64, mu, lam, area)) / (2 * h)
        np.testing.assert_allclose(g_ref, fd, rtol=0, atol=1e-5 * scale_g + 1e-9)


def _angle64(P):
    P0, P1, P2, P3 = P
    n1 = np.cross(P1 - P2, P0 - P2)
    n2 = np.cross(P0 - P3, P1 - P3)
    c = n1 @ n2 / np.sqrt((n1 @ n1) * (n2 @ n2))
    return np.sign(np.cross(n2, n1) @ (P1 - P0)) * np.arccos(np.clip(c, -1, 1))


def test_dihedral_oracle_matches_angle_and_its_derivative():
    rng = np.random.default_rng(3)
    for _ in range(50):
        P = rng.normal(0, 0.01, (4, 3)).astype(np.float32)
        th, g = O.dihedral(*P)
        P64 = P.astype(np.float64)
        assert abs(th - _angle64(P64)) < 2e-4
        h = 1e-8
        fd = np.zeros((4, 3))
        for i in range(4):
            for k in range(3):
                a, b = P64.copy(), P64.copy()
                a[i, k] += h
                b[i, k] -= h
                fd[i, k] = (_angle64(a) - _angle64(b)) / (2 * h)
        np.testing.assert_allclose(g, fd, rtol=0, atol=2e-3 * np.abs(fd).max())


def _deformed(sc, seed, amp=2e-3):
    rng = np.random.default_rng(seed)
    x = sc.x.copy()
    x[:, :3] += rng.normal(0, amp, (sc.num_verts, 3)).astype(np.float32)
    x[sc.pinned.astype(bool), :3] = sc.x[sc.pinned.astype(bool), :3]
    return x


def test_material_energy_sums():
    sc = S.cloth_on_sphere(n=16)
    x = _deformed(sc, 0)
    xt = sc.x.copy()
    e = O.material_energy(sc, x, xt, sc.dt)
    x64, xt64 = x[:, :3].astype(np.float64), xt[:, :3].astype(np.float64)
    scale = np.where(sc.pinned.astype(bool), sc.dirichlet, 1.0)
    e_in = np.sum(scale * sc.mass * np.sum((x64 - xt64) ** 2, 1) / (2 * sc.dt ** 2))
    e_st = sum(_energy64(*x64[f[:3]], sc.stretch_dm_inv[k].astype(np.float64), sc.stretch_mu, sc.stretch_lambda,
                         float(sc.stretch_area[k])) for k, f in enumerate(sc.stretch_faces))
    d = np.array([_angle64(x64[s]) for s in sc.bending]) - sc.bending_rest_angle
    e_b = np.sum(0.5 * sc.bending_k * sc.bending_scaling * sc.bending_hbar * d * d)
    assert e[1] == 0.0  # no springs under BW98
    np.testing.assert_allclose(e[[0, 2, 3]], [e_in, e_st, e_b], rtol=2e-4)


def test_fill_equals_assembled_per_element_outputs():
    sc = S.cloth_on_sphere(n=12)
    x = _deformed(sc, 1)
    xt = sc.x.copy()
    pat = N.MaterialPattern(sc)
    b, diag, (rp, col, val) = N.material_fill(sc, pat, x, xt, sc.dt)
    V = sc.num_verts
    # inertia alone
    sc0 = S.cloth_on_sphere(n=12)
    sc0.stretch_model, sc0.bending_model = 1, 0
    sc0.stretch_faces = sc0.stretch_faces[:0]
    b0, diag0, _ = N.material_fill(sc0, N.MaterialPattern(sc0), x, xt, sc.dt)
    B = b0[:, :3].astype(np.float64).copy()
    D = np.transpose(diag0[:, :, :3], (0, 2, 1)).astype(np.float64).copy()  # [v, row, col]
    dense = {}

    def add(r, c, blk):
        if r == c:
            D[r] += blk
        else:
            dense[(r, c)] = dense.get((r, c), 0) + blk

    ml = np.tile(np.float32([sc.stretch_mu, sc.stretch_lambda]), (sc.stretch_faces.shape[0], 1))
    g, h = O.eval_stretch_faces(x, sc.stretch_faces, sc.stretch_dm_inv, sc.stretch_area, ml)
    pairs3 = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)]
    for k, f in enumerate(sc.stretch_faces[:, :3]):
        for a in range(3):
            B[f[a]] -= g[k, a, :3]
        for m, (i, j) in enumerate(pairs3):
            add(f[i], f[j], h[k, m, :, :3].T)
    k_b = np.full(sc.bending.shape[0], sc.bending_k, np.float32)
    g, h = O.eval_bending(x, sc.bending, sc.bending_rest_angle, sc.bending_hbar, k_b, sc.bending_scaling)
    pairs4 = [(i, i) for i in range(4)] + [(i, j) for i in range(4) for j in range(4) if i != j]
    for k, s in enumerate(sc.bending):
        for a in range(4):
            B[s[a]] -= g[k, a, :3]
        for m, (i, j) in enumerate(pairs4):
            add(s[i], s[j], h[k, m, :, :3].T)
    np.testing.assert_allclose(b[:, :3], B, rtol=0, atol=1e-5 * np.abs(B).max())
    np.testing.assert_allclose(np.transpose(diag[:, :, :3], (0, 2, 1)), D, rtol=0, atol=1e-5 * np.abs(D).max())
    got = {}
    for r in range(V):
        for k in range(rp[r], rp[r + 1]):
            got[(r, int(col[k]))] = val[k].reshape(3, 3).T
    assert set(got) >= set(dense)
    smax = max(np.abs(v).max() for v in dense.values())
    for key, blk in dense.items():
        np.testing.assert_allclose(got[key], blk, rtol=0, atol=1e-5 * smax)
