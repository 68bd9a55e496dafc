"""Seeded contact configurations for the parity tests (positions only; meshes from scenes.py)."""
from __future__ import annotations

import os

import numpy as np

from luisacomputesimulator_b200 import scenes as S


def cloth_touching_sphere(gap=5e-4, seed=0, n=64):
    """Config-1 mesh with the cloth lowered until its lowest point is `gap` above the sphere top."""
    sc = S.cloth_on_sphere(n=n, seed=seed)
    x = sc.x.copy()
    nc = n * n
    cloth_min = x[:nc, 1].min()
    x[:nc, 1] += (0.2 + gap) - cloth_min
    return sc, x


def folded_cloth(n=48, gap=4e-4, seed=1):
    """A cloth folded over itself: the half with x > 0 mirrored onto a layer `gap` above."""
    cx, cf = S.cloth_grid(n, n, 0.01, jitter=1e-4, seed=seed)
    x = cx.astype(np.float64)
    right = x[:, 0] > 0
    x[right, 0] = -x[right, 0]
    x[right, 1] = x[right, 1] + gap + 0.002 * np.abs(x[right, 0])
    sc = S.assemble("folded", [S.MeshPart(cx, cf, np.zeros(cx.shape[0], bool))], dt=1 / 60, gravity=(0, -9.8, 0),
                    kappa=1e7)
    x4 = sc.x.copy()
    x4[:, :3] = x.astype(np.float32)
    return sc, x4


def random_motion(x, scale, seed):
    rng = np.random.default_rng(seed)
    out = x.copy()
    out[:, :3] += rng.normal(0.0, scale, (x.shape[0], 3)).astype(np.float32)
    return out


def twisted_tube_state(angle=1.2, n_around=300, n_along=296):
    """Config-2 tube with ring j rotated by angle * (2 j / (n_along - 1) - 1) about the x axis."""
    sc = S.twisted_tube(n_around, n_along)
    x = sc.x.copy()
    j = np.arange(sc.num_verts) // n_around
    ang = angle * (2.0 * j / (n_along - 1) - 1.0)
    c, s = np.cos(ang), np.sin(ang)
    y, z = x[:, 1].astype(np.float64), x[:, 2].astype(np.float64)
    x[:, 1] = (c * y - s * z).astype(np.float32)
    x[:, 2] = (s * y + c * z).astype(np.float32)
    return sc, x


TUBE_STATE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tube88k_state.npz")


def tube_state(path=TUBE_STATE):
    """Config-2 tube (300 x 296) at the state its run from rest reaches after `frame` steps, stepped by the
    CPU restatement (tests/golden/make_tube_state.py): (scene, x (V, 4), v (V, 4), frame), float32."""
    z = np.load(path)
    sc = S.twisted_tube(300, 296)
    x = sc.x.copy()
    x[:, :3] = z["x"]
    v = np.zeros_like(x)
    v[:, :3] = z["v"]
    return sc, x, v, int(z["frame"])


def sorted_pairs(p):
    p = np.asarray(p, np.int64).reshape(-1, 2)
    if len(p) == 0:
        return p
    return p[np.lexsort((p[:, 1], p[:, 0]))]
