"""One Newton iteration of the contact-and-solve path on the CPU, composed from the oracle.

TEST INFRASTRUCTURE ONLY: the timed CPU baseline of bench.py (``cpu_baseline`` and the
``--impl reference`` arm) and a checker for the GPU Newton loop.  It follows the loop body of
NewtonSolver::physics_step_GPU (Solver/SimulationSolver/newton_solver.cpp:4186-4284):
inertia + the cloth material (BW98 stretch and dihedral bending by default), contact set (LBVH build / refit / VF + EE queries,
barrier DCD), contact assembly, Jacobi-PCG, CCD line search, apply.
"""
from __future__ import annotations

import time

import numpy as np

from oracle import oracle as O


class MaterialPattern:
    """Fixed off-diagonal block pattern of the material elements (set-up, not timed): springs (both
    directions) for the spring model, the 6 ordered vertex pairs of each stretch face for BW98, the 12
    ordered pairs of each bending stencil unless bending is off; slots = block index of each contribution."""

    def __init__(self, sc):
        V = sc.num_verts
        e = sc.edges.astype(np.int64) if sc.stretch_model == 0 else np.zeros((0, 2), np.int64)
        f = sc.stretch_faces[:, :3].astype(np.int64) if sc.stretch_model == 1 else np.zeros((0, 3), np.int64)
        st = sc.bending.astype(np.int64) if sc.bending_model != 0 else np.zeros((0, 4), np.int64)
        dof = (sc.body_dof.astype(np.int64)[:, None] + np.arange(4)[None]) if sc.num_bodies else np.zeros((0, 4), np.int64)
        sk = np.stack([e[:, 0] * V + e[:, 1], e[:, 1] * V + e[:, 0]], 1).reshape(-1)
        fk = np.stack([f[:, i] * V + f[:, j] for i in range(3) for j in range(3) if i != j], 1).reshape(-1)
        bk = np.stack([st[:, i] * V + st[:, j] for i in range(4) for j in range(4) if i != j], 1).reshape(-1)
        ak = np.stack([dof[:, i] * V + dof[:, j] for i in range(4) for j in range(4) if i != j], 1).reshape(-1)
        uk = np.unique(np.concatenate([sk, fk, bk, ak]))
        self.nnz = len(uk)
        rp = np.zeros(V + 1, np.int64)
        np.add.at(rp, (uk // V) + 1, 1)
        self.rp = np.cumsum(rp).astype(np.uint32)
        self.col = (uk % V).astype(np.uint32)
        self.spring_slots = np.searchsorted(uk, sk).astype(np.uint32)
        self.face_slots = np.searchsorted(uk, fk).astype(np.uint32)
        self.bend_slots = np.searchsorted(uk, bk).astype(np.uint32)
        self.body_slots = np.searchsorted(uk, ak).astype(np.uint32)


def material_fill(sc, pat, x, x_tilde, dt):
    """orc_material_fill2: inertia (+ Dirichlet pinning) and the scene's stretch and bending models,
    b = -grad, diagonal (V, 3, 4) float4 columns, off-diagonal BSR on the fixed pattern."""
    V = sc.num_verts
    b = np.zeros((V, 4), np.float32)
    diag = np.zeros((V, 3, 4), np.float32)
    val = np.zeros((max(pat.nnz, 1), 9), np.float32)
    c = np.ascontiguousarray
    one = lambda a: a if a.size else np.zeros(1, a.dtype)  # noqa: E731
    per = [_opt(sc.stretch_mu_lambda), _opt(sc.bending_stiffness), _opt(sc.spring_stiffness)]  # kept alive
    O.lib().orc_material_fill2(
        V, O._p(O.f4(x)), O._p(c(sc.x, np.float32)), O._p(O.f4(x_tilde)), O._p(c(sc.mass, np.float32)),
        O._p(c(sc.pinned, np.uint8)), float(dt), float(sc.dirichlet), int(sc.stretch_model), int(sc.bending_model),
        sc.edges.shape[0], O._p(c(sc.edges, np.uint32)), O._p(c(sc.rest_len, np.float32)), float(sc.spring_k),
        sc.stretch_faces.shape[0], O._p(one(c(sc.stretch_faces, np.uint32))),
        O._p(one(c(sc.stretch_dm_inv, np.float32))), O._p(one(c(sc.stretch_area, np.float32))), float(sc.stretch_mu),
        float(sc.stretch_lambda), sc.bending.shape[0], O._p(one(c(sc.bending, np.uint32))),
        O._p(one(c(sc.bending_Q.reshape(-1, 16), np.float32))), O._p(one(c(sc.bending_rest_angle, np.float32))),
        O._p(one(c(sc.bending_hbar, np.float32))), float(sc.bending_k), float(sc.bending_scaling),
        O._p(one(pat.spring_slots)), O._p(one(pat.face_slots)), O._p(one(pat.bend_slots)), pat.nnz, O._p(b),
        O._p(diag), O._p(val), *[None if a is None else O._p(a) for a in per])
    if sc.num_bodies:  # rigid mesh rows inert, DOF slot rows from the bodies (orc_abd_fill)
        rigid, slot = rigid_mask(sc)
        b[rigid | slot] = 0.0
        diag[rigid | slot] = 0.0
        diag[rigid, 0, 0] = diag[rigid, 1, 1] = diag[rigid, 2, 2] = 1.0
        O.lib().orc_abd_fill(sc.num_bodies, O._p(c(sc.body_dof, np.uint32)),
                             O._p(c(sc.body_mass.reshape(-1, 16), np.float32)), O._p(c(sc.body_volume, np.float32)),
                             O._p(c(sc.body_kappa, np.float32)), O._p(body_fixed(sc)), O._p(O.f4(x)),
                             O._p(O.f4(x_tilde)), float(dt), float(sc.dirichlet), O._p(pat.body_slots), O._p(b),
                             O._p(diag), O._p(val))
    return b, diag, (pat.rp, pat.col, val[: pat.nnz])


def rigid_mask(sc):
    """(rigid mesh vertices, DOF slots) as boolean masks."""
    slot = np.zeros(sc.num_verts, bool)
    if sc.num_bodies:
        slot[(sc.body_dof.astype(np.int64)[:, None] + np.arange(4)[None]).ravel()] = True
    rigid = (sc.body != 0xFFFFFFFF) & ~slot
    return rigid, slot


def body_fixed(sc):
    rigid, _ = rigid_mask(sc)
    fixed = np.zeros(sc.num_bodies, np.uint8)
    sel = rigid & (sc.pinned != 0)
    fixed[sc.body[sel]] = 1
    return fixed


def affine_step(sc, x0, dx, alpha, out):
    """Rigid mesh vertices of out = p + A x_bar with q = q0 + alpha dq (the device's operation order)."""
    rigid, _ = rigid_mask(sc)
    if not rigid.any():
        return out
    f = np.float32
    a = f(alpha)
    d = sc.body_dof.astype(np.int64)[sc.body[rigid].astype(np.int64)]
    q = [x0[d + j, :3] + a * dx[d + j, :3] for j in range(4)]
    m = sc.model_x[rigid, :3]
    out[rigid, :3] = ((q[1] * m[:, 0:1] + q[2] * m[:, 1:2]) + q[3] * m[:, 2:3]) + q[0]
    return out


def affine_expand(sc, dx):
    """dx of rigid mesh vertices = J(x_bar) dq (k_abd_expand)."""
    rigid, _ = rigid_mask(sc)
    if rigid.any():
        d = sc.body_dof.astype(np.int64)[sc.body[rigid].astype(np.int64)]
        q = [dx[d + j, :3] for j in range(4)]
        m = sc.model_x[rigid, :3]
        dx[rigid, :3] = ((q[1] * m[:, 0:1] + q[2] * m[:, 1:2]) + q[3] * m[:, 2:3]) + q[0]
    return dx


def _opt(a):
    """an optional per-element array (None or empty: the scalar), contiguous float32"""
    return None if a is None or len(a) == 0 else np.ascontiguousarray(a, np.float32)


def material_system(sc, x, x_tilde, dt):
    """material_fill on a freshly built pattern."""
    return material_fill(sc, MaterialPattern(sc), x, x_tilde, dt)


def newton_iteration(sc, x, x_tilde, dt, timings=None, pattern=None, pcg_max_iter=100, pcg_rel_tol=1e-4,
                     pcg_check_every=25, info=None):
    """One CPU Newton iteration from positions x; returns (new x, toi, pcg stats, counts).

    The PCG stops at pcg_max_iter iterations, or when r.z < 1e-10 or |r| <= pcg_rel_tol |r0| at an
    iteration that is a multiple of pcg_check_every (the reference checks r.z every 25 iterations,
    precond_cg.cpp:681-755).  ``info`` (a dict), when given, receives the direction ``dx`` and the
    iterate ``x_iter`` the step bound was taken on."""
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
    if sc.num_bodies:
        b, diag = O.contact_grad_diag_abd(pairs, sc, b, diag)
        B = O.contact_offdiag_bsr_abd(pairs, sc)
    else:
        b, diag = O.contact_grad_diag(pairs, sc.num_verts, b, diag)
        B = O.contact_offdiag_bsr(pairs, sc.num_verts)
    c3 = time.perf_counter()
    dx, st = O.pcg(diag, A, B, b, max_iter=pcg_max_iter, rel_tol=pcg_rel_tol, abs_rz_tol=1e-10,
                   check_every=pcg_check_every)
    c4 = time.perf_counter()
    dx = affine_expand(sc, dx)
    x1 = x.copy()
    x1[:, :3] += dx[:, :3]
    x1 = affine_step(sc, x, dx, 1.0, x1)
    O.lbvh_refit(tf, x, x1, sc.faces, sc.offset)
    O.lbvh_refit(te, x, x1, sc.edges, sc.offset)
    cvf, _ = O.lbvh_query_vf(tf, x, x1, sc.d_hat, sc.offset)
    cee, _ = O.lbvh_query_ee(te, x, x1, sc.edges, sc.d_hat, sc.offset)
    g1, _ = O.ccd_vf(cvf, x, x1, sc.faces, sc.body, sc.offset, per_pair=False)
    g2, _ = O.ccd_ee(cee, x, x1, sc.edges, sc.body, sc.offset, per_pair=False)
    toi = min(g1, g2)
    out = x.copy()
    out[:, :3] += np.float32(toi) * dx[:, :3]
    out = affine_step(sc, x, dx, toi, out)
    c5 = time.perf_counter()
    for k, v in dict(material=c1 - c0, dcd_broad=c2 - c1, dcd_narrow_assembly=c3 - c2, pcg=c4 - c3,
                     ccd=c5 - c4).items():
        t[k] = t.get(k, 0.0) + v
    if info is not None:
        info.update(dx=dx, x_iter=x, ccd_vf=len(cvf), ccd_ee=len(cee))
    return out, toi, st, dict(vf=n_vf, ee=n_ee, pairs=len(pairs))


# ------------------------------------------------------------------------------------ time step
_F = np.float32


def pinned_targets(sc, t):
    """Targets of the animated pinned vertices at time t (float32), in the order of the device's
    k_targets: scale, rotation about an axis through a centre (Rodrigues), translation
    (WorldData::get_fixed_point_target_positions, Solver/Initializer/init_mesh_data.cpp:272-297).
    cos/sin are numpy's float32 functions, which may differ from CUDA's cosf/sinf in the last bit."""
    p = sc.x[:, :3].astype(np.float32).copy()
    t = _F(t)
    for an in sc.anims:
        vids, center, axis, omega = an[:4]
        translate, scale, mode = (an[4], an[5], an[6]) if len(an) > 4 else (None, None, 1)
        q = p[vids]
        if mode & 2:
            q = (np.asarray(scale, np.float32) * t) * q
        if mode & 1:
            ax = np.asarray(axis, np.float64)
            n = np.linalg.norm(ax)
            ax = (ax / n if n > 0 else ax).astype(np.float32)
            c3 = np.asarray(center, np.float32)
            ang = _F(omega) * t
            c, s = np.cos(ang, dtype=np.float32), np.sin(ang, dtype=np.float32)
            px, py, pz = q[:, 0] - c3[0], q[:, 1] - c3[1], q[:, 2] - c3[2]
            d = (ax[0] * px + ax[1] * py) + ax[2] * pz
            kx, ky, kz = ax[1] * pz - ax[2] * py, ax[2] * px - ax[0] * pz, ax[0] * py - ax[1] * px
            omc = _F(1.0) - c
            q = np.stack([((c3[0] + px * c) + kx * s) + (ax[0] * d) * omc,
                          ((c3[1] + py * c) + ky * s) + (ax[1] * d) * omc,
                          ((c3[2] + pz * c) + kz * s) + (ax[2] * d) * omc], 1).astype(np.float32)
        if mode & 4:
            q = q + np.asarray(translate, np.float32) * t
        p[vids] = q
    return p


def step_time(frame, dt):
    """The time the step after `frame` steps animates to: the device keeps a double clock advanced by the
    float dt at the start of every step and passes it to the targets as a float."""
    return np.float32(frame * float(np.float32(dt)) + float(np.float32(dt)))


def predict(sc, x, v, t):
    """fn_predict_position (Solver/SimulationSolver/newton_solver.cpp:576-604) with the pinned vertices'
    velocity set towards their targets (physics_step_prev_operation, solver_interface.cpp:130-162):
    returns (x_tilde, v) as float32 (V, 4)."""
    dt = _F(sc.dt)
    g = np.asarray(sc.gravity, np.float32)
    v = v.astype(np.float32).copy()
    pin = sc.pinned.astype(bool)
    tg = pinned_targets(sc, t)
    v[pin, :3] = (tg[pin] - x[pin, :3]) / dt
    vp = v[:, :3] + dt * g
    vp[pin] = v[pin, :3]
    xt = x.astype(np.float32).copy()
    xt[:, :3] = x[:, :3] + dt * vp
    xt[:, 3] = 0.0
    return xt, v


def floor_ccd(x0, x1, offset, pinned, floor_y):
    """fn_gound_collision_ccd (Solver/SimulationSolver/newton_solver.cpp:952-1000): every free vertex whose
    end position minus its offset lies below the floor bounds the step by
    (y0 - offset - floor_y) / (y0 - y1) / 1.25 (accd::line_search_max_t); the minimum of those, 1 when none."""
    f = np.float32
    off = np.asarray(offset, f)
    y0, y1 = x0[:, 1].astype(f), x1[:, 1].astype(f)
    sel = ~np.asarray(pinned, bool) & ((y1 - off) < f(floor_y))
    if not sel.any():
        return 1.0
    toi = ((y0[sel] - off[sel]) - f(floor_y)) / (y0[sel] - y1[sel]) / f(1.25)
    return float(toi.min())


def time_step(sc, x, v, frame, pattern=None, nonlinear_iters=3, pcg_max_iter=100, pcg_rel_tol=1e-4,
              pcg_check_every=25, damping=2.0, log=None):
    """One time step of NewtonSolver::physics_step_GPU (newton_solver.cpp:4152-4297) for soft scenes
    without a floor: predict, Newton iterations until the direction is small (max |dx| < 1e-2 dt) or,
    after `nonlinear_iters` iterations, the pinned vertices are within 1e-3 of their targets
    (line_search, newton_solver.cpp:3784-3880), then the damped velocity update
    (fn_update_velocity, newton_solver.cpp:606-633).  Returns (x, v, per-iteration records)."""
    if sc.num_bodies:
        raise ValueError("time_step: affine bodies are not restated here")
    pat = pattern if pattern is not None else MaterialPattern(sc)
    dt = _F(sc.dt)
    x = x.astype(np.float32).copy()
    x_step = x.copy()
    xt, v = predict(sc, x, v, step_time(frame, sc.dt))
    pin = sc.pinned.astype(bool)
    recs = [] if log is None else log
    glob = dirich = False
    for it in range(100):
        if glob or (it >= nonlinear_iters and dirich):
            break
        info = {}
        x, toi, st, cnt = newton_iteration(sc, x, xt, dt, pattern=pat, pcg_max_iter=pcg_max_iter,
                                           pcg_rel_tol=pcg_rel_tol, pcg_check_every=pcg_check_every, info=info)
        d = info["dx"][:, :3]
        max_dx = float(np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).max(initial=0.0))
        e = x[pin, :3] - xt[pin, :3]
        dirichlet = float(np.sqrt((e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1]) + e[:, 2] * e[:, 2]).max(initial=0.0))
        glob = max_dx < float(_F(1e-2) * dt)
        dirich = dirichlet < 1e-3
        recs.append(dict(toi=float(toi), pcg_iters=st["iterations"], rel_residual=st["rel_residual"],
                         max_dx=max_dx, dirichlet=dirichlet, ccd_vf=info["ccd_vf"], ccd_ee=info["ccd_ee"], **cnt))
    f = np.exp(_F(-damping) * dt, dtype=np.float32)
    v = np.zeros_like(x)
    v[:, :3] = (x[:, :3] - x_step[:, :3]) / dt * f
    return x, v, recs
