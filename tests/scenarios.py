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


def deep_tree_elements(kind, dup_top=8):
    """Elements whose sorted Morton codes make an LBVH with inner nodes deeper than 32 levels, where the
    reference's 32-entry traversal stack can fill up: for every bit k of the 30-bit code, two elements whose
    code has every bit but k set (each such pair becomes an inner node to the left of all larger codes, so a
    traversal keeps one pending node per level), `dup_top` elements at the all-ones code and one at code 0.
    The elements at code 0 and at the top reach the corners 0 and 1024 of the global box, so a centre
    quantises to the integer part of its coordinates.  kind "face": degenerate triangles, kind "edge":
    degenerate edges.  Returns (x (V, 4) float32, elements (n, 4 | 2) uint32)."""
    m = 3 if kind == "face" else 2
    elems = []
    for k in range(30):
        axis, bit = 2 - k % 3, k // 3  # Morton bit 3 j + 2 is x bit j, 3 j + 1 is y bit j, 3 j is z bit j
        c = np.full(3, 1023.5)
        c[axis] -= 2 ** bit
        elems += [[c - 0.25, c + 0.25, c][:m]] * 2
    top = np.full(3, 1023.5)
    elems.append([top - 0.5, top + 0.5, top][:m])  # reaches 1024
    elems += [[top - 0.25, top + 0.25, top][:m]] * (dup_top - 1)
    elems.append([np.zeros(3), np.ones(3), np.full(3, 0.5)][:m])  # reaches 0
    x = np.zeros((len(elems) * m, 4), np.float32)
    x[:, :3] = np.asarray([v for e in elems for v in e], np.float64).astype(np.float32)
    el = np.arange(len(elems) * m, dtype=np.uint32).reshape(-1, m)
    if kind == "face":  # faces are stored as uint4 (the layout of Buffer<uint3>)
        el = np.concatenate([el, np.zeros((len(el), 1), np.uint32)], 1)
    return x, el


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
