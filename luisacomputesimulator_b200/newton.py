"""Host-side mirror of NewtonSolver (Solver/SimulationSolver/newton_solver.h:29-51) over the C ABI:
``NewtonSolver(scene).physics_step_GPU()`` advances one time step on the device."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi as A


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def scene_desc(sc, keep, nonlinear_iters=3, pcg_max_iter=100, pcg_rel_tol=1e-4, pcg_abs_rz_tol=1e-10,
               pcg_check_every=25, damping=2.0, use_floor=False, floor_y=0.0):
    """lcs_scene_desc of a scene (host arrays appended to `keep`, which must outlive the call that reads it)."""
    def arr(a, dtype):
        a = _c(a, dtype)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    d = A.SceneDesc()
    d.n_verts, d.n_faces, d.n_edges, d.n_bending = sc.num_verts, sc.faces.shape[0], sc.edges.shape[0], \
        sc.bending.shape[0]
    d.x = arr(sc.x, np.float32)
    d.v = None
    d.faces = arr(sc.faces, np.uint32)
    d.edges = arr(sc.edges, np.uint32)
    d.bending = arr(sc.bending, np.uint32)
    d.bending_Q = arr(sc.bending_Q.reshape(-1, 16), np.float32)
    d.rest_len = arr(sc.rest_len, np.float32)
    d.vert_area = arr(sc.vert_area, np.float32)
    d.face_area = arr(sc.face_area, np.float32)
    d.edge_area = arr(sc.edge_area, np.float32)
    d.mass = arr(sc.mass, np.float32)
    d.d_hat = arr(sc.d_hat, np.float32)
    d.offset = arr(sc.offset, np.float32)
    d.body = arr(sc.body, np.uint32)
    d.pinned = arr(sc.pinned, np.uint8)
    groups = np.full(sc.num_verts, -1, np.int8)
    anim = np.zeros((max(len(sc.anims), 1), 16), np.float32)
    for gi, an in enumerate(sc.anims):
        vids, center, axis, omega = an[:4]
        translate, scale, mode = (an[4], an[5], an[6]) if len(an) > 4 else (None, None, 1)
        groups[vids] = gi
        ax = np.asarray(axis, np.float64)
        n_ax = np.linalg.norm(ax)
        anim[gi, :3] = center
        anim[gi, 3:6] = ax / n_ax if n_ax > 0 else 0.0
        anim[gi, 6] = omega
        anim[gi, 7] = mode
        if translate is not None:
            anim[gi, 8:11] = translate
        if scale is not None:
            anim[gi, 11:14] = scale
    d.anim_group = arr(groups, np.int8)
    d.n_anim = len(sc.anims)
    d.anim = arr(anim, np.float32)
    d.dt = sc.dt
    d.gravity = (C.c_float * 3)(*sc.gravity)
    d.kappa, d.spring_k, d.bending_k, d.dirichlet, d.damping = sc.kappa, sc.spring_k, sc.bending_k, \
        sc.dirichlet, damping
    d.use_floor, d.floor_y = int(use_floor), floor_y
    d.nonlinear_iters, d.pcg_max_iter = nonlinear_iters, pcg_max_iter
    d.pcg_rel_tol, d.pcg_abs_rz_tol, d.pcg_check_every = pcg_rel_tol, pcg_abs_rz_tol, pcg_check_every
    d.stretch_model, d.bending_model = sc.stretch_model, sc.bending_model
    d.n_stretch_faces = sc.stretch_faces.shape[0]
    d.stretch_faces = arr(sc.stretch_faces, np.uint32)
    d.stretch_dm_inv = arr(sc.stretch_dm_inv, np.float32)
    d.stretch_area = arr(sc.stretch_area, np.float32)
    d.stretch_mu, d.stretch_lambda = sc.stretch_mu, sc.stretch_lambda
    d.bending_rest_angle = arr(sc.bending_rest_angle, np.float32)
    d.bending_hbar = arr(sc.bending_hbar, np.float32)
    d.bending_scaling = sc.bending_scaling
    if sc.stretch_mu_lambda is not None:
        d.stretch_mu_lambda = arr(sc.stretch_mu_lambda, np.float32)
    if sc.bending_stiffness is not None:
        d.bending_stiffness = arr(sc.bending_stiffness, np.float32)
    if sc.spring_stiffness is not None:
        d.spring_stiffness = arr(sc.spring_stiffness, np.float32)
    d.n_bodies = sc.num_bodies
    if sc.num_bodies:
        d.body_dof = arr(sc.body_dof, np.uint32)
        d.body_mass = arr(sc.body_mass.reshape(-1, 16), np.float32)
        d.body_volume = arr(sc.body_volume, np.float32)
        d.body_kappa = arr(sc.body_kappa, np.float32)
        d.model_x = arr(sc.model_x, np.float32)
    return d


class NewtonSolver:
    """One scene, state resident on the device.

    plain=True selects the reference's dispatch structure (the one-scene comparator);
    fp64=True the precision form; profile=True per-phase CUDA-event timing;
    single_reduction=True the single-reduction row-resident PCG (fused mode; slice-resident where the rows fit,
    unless global_matrix=True); energy_linesearch=True the
    reference's use_energy_linesearch (step halving until the energy decreases).
    """

    def __init__(self, scene, plain=False, fp64=False, profile=False, nonlinear_iters=3, pcg_max_iter=100,
                 pcg_rel_tol=1e-4, pcg_abs_rz_tol=1e-10, pcg_check_every=25, damping=2.0, use_floor=False,
                 floor_y=0.0, stream=None, single_reduction=False, full_traversal=False, energy_linesearch=False,
                 global_matrix=False, deterministic=False):
        self.lib = A.load()
        self.scene = scene
        sc = scene
        self._keep = []

        d = scene_desc(sc, self._keep, nonlinear_iters, pcg_max_iter, pcg_rel_tol, pcg_abs_rz_tol,
                       pcg_check_every, damping, use_floor, floor_y)
        self.desc = d
        flags = (A.LCS_NEWTON_PLAIN if plain else 0) | (A.LCS_NEWTON_FP64 if fp64 else 0) | \
            (A.LCS_NEWTON_PROFILE if profile else 0) | (A.LCS_NEWTON_PCG_SINGLE_REDUCTION if single_reduction else 0) | \
            (A.LCS_NEWTON_FULL_TRAVERSAL if full_traversal else 0) | \
            (A.LCS_NEWTON_ENERGY_LINESEARCH if energy_linesearch else 0) | \
            (A.LCS_NEWTON_PCG_GLOBAL_MATRIX if global_matrix else 0) | \
            (A.LCS_NEWTON_DETERMINISTIC if deterministic else 0)
        s = C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        h = C.c_void_p()
        A.check(self.lib.lcs_newton_create(C.byref(d), flags, s, C.byref(h)), "lcs_newton_create")
        self.h = h
        self.plain, self.fp64 = plain, fp64
        self.stats = A.NewtonStats()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lcs_newton_destroy(self.h)
            self.h = None

    def physics_step_GPU(self):
        A.check(self.lib.lcs_newton_step(self.h, C.byref(self.stats)), "lcs_newton_step")
        return self.stats

    step = physics_step_GPU

    def step_host(self, x_in=None, v_in=None, x_out=None, v_out=None):
        p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        A.check(self.lib.lcs_newton_step_host(self.h, p(x_in), p(v_in), p(x_out), p(v_out), C.byref(self.stats)),
                "lcs_newton_step_host")
        return self.stats

    def invalidate(self):
        """Announce positions written through state_ptrs() (the next step re-traverses for its DCD lists)."""
        A.check(self.lib.lcs_newton_invalidate(self.h), "lcs_newton_invalidate")

    def state_ptrs(self):
        x, v = C.c_void_p(), C.c_void_p()
        A.check(self.lib.lcs_newton_state(self.h, C.byref(x), C.byref(v)), "lcs_newton_state")
        return x.value, v.value

    def positions(self):
        """Copy of the device positions, float32 (V, 4); synchronises."""
        out = np.zeros((self.scene.num_verts, 4), np.float32)
        A.check(self.lib.lcs_newton_download(self.h, out.ctypes.data_as(C.c_void_p), None), "lcs_newton_download")
        return out

    def velocities(self):
        out = np.zeros((self.scene.num_verts, 4), np.float32)
        A.check(self.lib.lcs_newton_download(self.h, None, out.ctypes.data_as(C.c_void_p)), "lcs_newton_download")
        return out

    def upload(self, x=None, v=None):
        """Replace the device positions / velocities, float32 (V, 4) each (either may be None)."""
        p = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)  # noqa: E731
        xa, va = p(x), p(v)
        for a in (xa, va):
            if a is not None and a.shape != (self.scene.num_verts, 4):
                raise ValueError(f"state of shape {a.shape}, expected ({self.scene.num_verts}, 4)")
        q = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        A.check(self.lib.lcs_newton_upload(self.h, q(xa), q(va)), "lcs_newton_upload")

    def iteration_log(self):
        """Per-iteration records of the last step: dicts of pcg_iters, rel_residual, toi, max_dx and the
        DCD / CCD candidate and contact pair counts."""
        cap = 128
        recs = (A.IterRecord * cap)()
        n = C.c_int32()
        A.check(self.lib.lcs_newton_iteration_log(self.h, recs, cap, C.byref(n)), "lcs_newton_iteration_log")
        return [{f: getattr(recs[k], f) for f, _ in A.IterRecord._fields_} for k in range(min(n.value, cap))]

    def set_frame(self, frame):
        """Frame counter (the reference's current_frame): the next step animates the pins to (frame + 1) dt."""
        A.check(self.lib.lcs_newton_set_frame(self.h, int(frame)), "lcs_newton_set_frame")

    def frame(self):
        f = C.c_uint32()
        A.check(self.lib.lcs_newton_get_frame(self.h, C.byref(f)), "lcs_newton_get_frame")
        return int(f.value)

    def save_current_frame_state_to_host(self, path):
        """The reference's frame state file (positions, velocities, body q and q velocities) for this state."""
        from . import scene_io
        scene_io.save_state(path, self.scene, self.positions(), self.velocities())

    def load_saved_state_from_host(self, path):
        """Load a frame state file written by the reference or by save_current_frame_state_to_host."""
        from . import scene_io
        x, v = scene_io.load_state(path, self.scene, self.positions())
        self.upload(x, v)

    def last_iterate(self):
        """(x at the start of the last Newton iteration, its direction dx, x_tilde), float32 (V, 4) each."""
        out = [np.zeros((self.scene.num_verts, 4), np.float32) for _ in range(3)]
        A.check(self.lib.lcs_newton_last_iterate(self.h, *[o.ctypes.data_as(C.c_void_p) for o in out]),
                "lcs_newton_last_iterate")
        return tuple(out)

    def profile(self):
        ms = (C.c_double * 9)()
        n = (C.c_int32 * 9)()
        A.check(self.lib.lcs_newton_profile(self.h, ms, n, 9), "lcs_newton_profile")
        return {A.PHASES[i]: (ms[i], n[i]) for i in range(9)}

    def reset_profile(self):
        A.check(self.lib.lcs_newton_reset_profile(self.h), "lcs_newton_reset_profile")

    def pcg_kind(self):
        """'plain', 'fused' (persistent CSR solve), 'rows', 'cg1' (row-resident: classic, single-reduction) or
        'cg1-res' (single-reduction, slice-resident: one block per SM with its matrix groups in shared memory)."""
        return ["plain", "fused", "rows", "cg1", "cg1-res"][self.lib.lcs_newton_pcg_kind(self.h)]

    def uses_row_pcg(self):
        return self.pcg_kind() in ("rows", "cg1", "cg1-res")

    def counts(self):
        v = [C.c_uint32() for _ in range(4)]
        A.check(self.lib.lcs_newton_counts(self.h, *[C.byref(a) for a in v]), "lcs_newton_counts")
        return dict(nnz_material=v[0].value, cap_vf=v[1].value, cap_ee=v[2].value, cap_pairs=v[3].value)


class NewtonBatch:
    """Many independent scenes stepped together (lcs_newton_create_batch): one set of launches per
    Newton phase for all scenes, per-scene trees, step bounds and PCG (one thread-block cluster of
    `cluster` CTAs per scene).  A scene's trajectory does not depend on the other scenes: with
    deterministic=True (the default when no scene has affine bodies) every sum runs in a fixed order, so a
    scene's result is bit-identical alone and in any mix (LCS_NEWTON_DETERMINISTIC)."""

    def __init__(self, scenes, fp64=False, profile=False, cluster=0, nonlinear_iters=3, pcg_max_iter=100,
                 pcg_rel_tol=1e-4, pcg_abs_rz_tol=1e-10, damping=2.0, stream=None, deterministic=None):
        self.lib = A.load()
        self.scenes = list(scenes)
        keep = []
        descs = (A.SceneDesc * len(self.scenes))()
        for k, sc in enumerate(self.scenes):
            descs[k] = scene_desc(sc, keep, nonlinear_iters, pcg_max_iter, pcg_rel_tol, pcg_abs_rz_tol, 1, damping)
        if deterministic is None:  # sums in a fixed order wherever the deterministic mode covers the scenes
            deterministic = all(sc.num_bodies == 0 for sc in self.scenes)
        self.deterministic = bool(deterministic)
        flags = (A.LCS_NEWTON_FP64 if fp64 else 0) | (A.LCS_NEWTON_PROFILE if profile else 0) | \
            (A.LCS_NEWTON_DETERMINISTIC if deterministic else 0)
        s = C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        h = C.c_void_p()
        A.check(self.lib.lcs_newton_create_batch(descs, len(self.scenes), flags, s, int(cluster), C.byref(h)),
                "lcs_newton_create_batch")
        self.h = h
        self.stats = A.NewtonStats()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lcs_newton_destroy(self.h)
            self.h = None

    def step(self):
        A.check(self.lib.lcs_newton_step(self.h, C.byref(self.stats)), "lcs_newton_step")
        return self.stats

    def pcg_tuning(self):
        """(chunks of 256 rows per CTA, solve ms) picked by the batched PCG's autotuner (0 before tuning)."""
        t, ms = C.c_uint32(), C.c_float()
        A.check(self.lib.lcs_newton_batch_tuning(self.h, C.byref(t), C.byref(ms)), "lcs_newton_batch_tuning")
        return int(t.value), float(ms.value)

    def query_tuning(self):
        """(VF, EE) threads per block picked by the traversal autotuner on the first step (0 before it)."""
        a, b = C.c_uint32(), C.c_uint32()
        A.check(self.lib.lcs_newton_batch_query_tuning(self.h, C.byref(a), C.byref(b)),
                "lcs_newton_batch_query_tuning")
        return int(a.value), int(b.value)

    def scene_stats(self, k):
        st = A.NewtonStats()
        A.check(self.lib.lcs_newton_scene_stats(self.h, k, C.byref(st)), "lcs_newton_scene_stats")
        return st

    def positions(self, k):
        out = np.zeros((self.scenes[k].num_verts, 4), np.float32)
        A.check(self.lib.lcs_newton_download_scene(self.h, k, out.ctypes.data_as(C.c_void_p), None),
                "lcs_newton_download_scene")
        return out

    def velocities(self, k):
        out = np.zeros((self.scenes[k].num_verts, 4), np.float32)
        A.check(self.lib.lcs_newton_download_scene(self.h, k, None, out.ctypes.data_as(C.c_void_p)),
                "lcs_newton_download_scene")
        return out

    def profile(self):
        ms = (C.c_double * 9)()
        n = (C.c_int32 * 9)()
        A.check(self.lib.lcs_newton_profile(self.h, ms, n, 9), "lcs_newton_profile")
        return {A.PHASES[i]: (ms[i], n[i]) for i in range(9)}

    def reset_profile(self):
        A.check(self.lib.lcs_newton_reset_profile(self.h), "lcs_newton_reset_profile")
