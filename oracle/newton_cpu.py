"""One Newton iteration of the contact-and-solve path on the CPU, composed from the oracle.

TEST INFRASTRUCTURE ONLY: the timed CPU baseline of bench.py (``cpu_baseline`` and the
``--impl reference`` arm) and a checker for the GPU Newton loop.  It follows the loop body of
NewtonSolver::physics_step_GPU (Solver/SimulationSolver/newton_solver.cpp:4186-4284):
inertia + springs + quadratic bending, contact set (LBVH build / refit / VF + EE queries,
barrier DCD), contact assembly, Jacobi-PCG, CCD line search, apply.
"""
from __future__ import annotations

import time

import numpy as np

from oracle import oracle as O


def material_system(sc, x, x_tilde, dt):
    """Inertia (+ Dirichlet pinning), springs and rest-relative quadratic bending:
    b = -grad, diag (V, 3, 4) column-major float4 columns, off-diagonal BSR."""
    V = sc.num_verts
    xv = x[:, :3].astype(np.float64)
    h2 = 1.0 / (dt * dt)
    m = sc.mass.astype(np.float64)
    scale = np.where(sc.pinned.astype(bool), 1.0 + sc.dirichlet, 1.0)
    b = -(m * h2 * scale)[:, None] * (xv - x_tilde[:, :3])
    D = np.zeros((V, 3, 3))
    D[:, 0, 0] = D[:, 1, 1] = D[:, 2, 2] = m * h2 * scale
    # springs (newton_solver.cpp:1003-1045)
    e = sc.edges.astype(np.int64)
    d = xv[e[:, 0]] - xv[e[:, 1]]
    l = np.maximum(np.linalg.norm(d, axis=1), 1.19209290e-7)
    L = sc.rest_len.astype(np.float64)
    k = sc.spring_k
    g = (k * (l - L) / l)[:, None] * d
    np.add.at(b, e[:, 0], -g)
    np.add.at(b, e[:, 1], g)
    xxT = d[:, :, None] * d[:, None, :] / (l * l)[:, None, None]
    H = k * xxT + (k * np.maximum(1 - L / l, 0))[:, None, None] * (np.eye(3)[None] - xxT)
    np.add.at(D, e[:, 0], H)
    np.add.at(D, e[:, 1], H)
    rows = [e[:, 0], e[:, 1]]
    cols = [e[:, 1], e[:, 0]]
    blocks = [-H, -H]
    # quadratic bending relative to rest (init_sim_data.cpp:455-480)
    st = sc.bending.astype(np.int64)
    Q = sc.bending_Q.astype(np.float64) * sc.bending_k
    u = xv[st] - sc.x[st][:, :, :3].astype(np.float64)  # (B, 4, 3)
    gb = np.einsum("bij,bjk->bik", Q, u)
    for i in range(4):
        np.add.at(b, st[:, i], -gb[:, i])
        np.add.at(D, st[:, i], Q[:, i, i][:, None, None] * np.eye(3)[None])
        for j in range(4):
            if i != j:
                rows.append(st[:, i])
                cols.append(st[:, j])
                blocks.append(Q[:, i, j][:, None, None] * np.eye(3)[None])
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    blocks = np.concatenate(blocks)
    key = rows * V + cols
    uk, inv = np.unique(key, return_inverse=True)
    val = np.zeros((len(uk), 3, 3))
    np.add.at(val, inv, blocks)
    rp = np.zeros(V + 1, np.int64)
    np.add.at(rp, (uk // V) + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    val9 = np.ascontiguousarray(np.transpose(val, (0, 2, 1)).reshape(-1, 9), np.float32)
    diag = np.zeros((V, 3, 4), np.float32)
    diag[:, :, :3] = np.transpose(D, (0, 2, 1))
    b4 = np.zeros((V, 4), np.float32)
    b4[:, :3] = b
    return b4, diag, (rp, (uk % V).astype(np.uint32), val9)


class MaterialPattern:
    """Fixed off-diagonal block pattern of springs + bending stencils (set-up, not timed)."""

    def __init__(self, sc):
        V = sc.num_verts
        e = sc.edges.astype(np.int64)
        st = sc.bending.astype(np.int64)
        rows = [e[:, 0], e[:, 1]]
        cols = [e[:, 1], e[:, 0]]
        sk = np.stack([e[:, 0] * V + e[:, 1], e[:, 1] * V + e[:, 0]], 1).reshape(-1)
        bk = []
        for i in range(4):
            for j in range(4):
                if i != j:
                    bk.append(st[:, i] * V + st[:, j])
        bk = np.stack(bk, 1).reshape(-1) if len(st) else np.zeros(0, np.int64)
        uk = np.unique(np.concatenate([sk, bk]))
        self.nnz = len(uk)
        rp = np.zeros(V + 1, np.int64)
        np.add.at(rp, (uk // V) + 1, 1)
        self.rp = np.cumsum(rp).astype(np.uint32)
        self.col = (uk % V).astype(np.uint32)
        self.spring_slots = np.searchsorted(uk, sk).astype(np.uint32)
        self.bend_slots = np.searchsorted(uk, bk).astype(np.uint32)
        del rows, cols


def material_fill(sc, pat, x, x_tilde, dt):
    """orc_material_fill: the C restatement of the material producers on the fixed pattern."""
    V = sc.num_verts
    b = np.zeros((V, 4), np.float32)
    diag = np.zeros((V, 3, 4), np.float32)
    val = np.zeros((pat.nnz, 9), np.float32)
    c = np.ascontiguousarray
    O.lib().orc_material_fill(V, sc.edges.shape[0], sc.bending.shape[0], O._p(O.f4(x)), O._p(c(sc.x, np.float32)),
                              O._p(O.f4(x_tilde)), O._p(c(sc.mass, np.float32)), O._p(c(sc.pinned, np.uint8)),
                              float(dt), float(sc.dirichlet), O._p(c(sc.edges, np.uint32)),
                              O._p(c(sc.rest_len, np.float32)), float(sc.spring_k), O._p(c(sc.bending, np.uint32)),
                              O._p(c(sc.bending_Q.reshape(-1, 16), np.float32)), float(sc.bending_k),
                              O._p(pat.spring_slots), O._p(pat.bend_slots), pat.nnz, O._p(b), O._p(diag), O._p(val))
    return b, diag, (pat.rp, pat.col, val)


def newton_iteration(sc, x, x_tilde, dt, timings=None, pattern=None):
    """One CPU Newton iteration from positions x; returns (new x, toi, pcg stats, counts)."""
    t = {} if timings is None else timings
    c0 = time.perf_counter()
    if pattern is None:
        b, diag, A = material_system(sc, x, x_tilde, dt)
    else:
        b, diag, A = material_fill(sc, pattern, x, x_tilde, dt)
    c1 = time.perf_counter()
    tf = O.lbvh_build(O.TREE_FACE, x, sc.faces, sc.num_verts)
    te = O.lbvh_build(O.TREE_EDGE, x, sc.edges, sc.num_verts)
    O.lbvh_refit(tf, x, x, sc.faces, sc.offset)
    O.lbvh_refit(te, x, x, sc.edges, sc.offset)
    vf, n_vf = O.lbvh_query_vf(tf, x, x, sc.d_hat, sc.offset)
    ee, n_ee = O.lbvh_query_ee(te, x, x, sc.edges, sc.d_hat, sc.offset)
    c2 = time.perf_counter()
    pairs = np.concatenate([
        O.dcd_vf(vf, x, sc.faces, sc.body, sc.vert_area, sc.face_area, sc.d_hat, sc.offset, sc.kappa),
        O.dcd_ee(ee, x, sc.edges, sc.body, sc.edge_area, sc.d_hat, sc.offset, sc.kappa)])
    b, diag = O.contact_grad_diag(pairs, sc.num_verts, b, diag)
    B = O.contact_offdiag_bsr(pairs, sc.num_verts)
    c3 = time.perf_counter()
    dx, st = O.pcg(diag, A, B, b, max_iter=100, rel_tol=1e-4, abs_rz_tol=1e-10, check_every=25)
    c4 = time.perf_counter()
    x1 = x.copy()
    x1[:, :3] += dx[:, :3]
    O.lbvh_refit(tf, x, x1, sc.faces, sc.offset)
    O.lbvh_refit(te, x, x1, sc.edges, sc.offset)
    cvf, _ = O.lbvh_query_vf(tf, x, x1, sc.d_hat, sc.offset)
    cee, _ = O.lbvh_query_ee(te, x, x1, sc.edges, sc.d_hat, sc.offset)
    g1, _ = O.ccd_vf(cvf, x, x1, sc.faces, sc.body, sc.offset, per_pair=False)
    g2, _ = O.ccd_ee(cee, x, x1, sc.edges, sc.body, sc.offset, per_pair=False)
    toi = min(g1, g2)
    out = x.copy()
    out[:, :3] += np.float32(toi) * dx[:, :3]
    c5 = time.perf_counter()
    for k, v in dict(material=c1 - c0, dcd_broad=c2 - c1, dcd_narrow_assembly=c3 - c2, pcg=c4 - c3,
                     ccd=c5 - c4).items():
        t[k] = t.get(k, 0.0) + v
    return out, toi, st, dict(vf=n_vf, ee=n_ee, pairs=len(pairs))
