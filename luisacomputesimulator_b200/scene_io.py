"""Scene ingestion: the reference's OBJ meshes and scene JSON files as Scenes for the Newton loop.

* ``read_obj``: vertex positions and triangles of a Wavefront OBJ, as the reference's
  ``read_mesh_file`` takes them (Solver/MeshOperation/mesh_reader.cpp:355-500): vertices in file order,
  the faces of every object/group in file order, polygons fanned into triangles (0, i, i + 1), faces with
  a repeated vertex dropped.
* ``load_scene_json``: the scene file format of ``load_scene_params_from_json``
  (Application/app_simulation_demo_config.cpp:49-766): scene parameters (implicit_dt, gravity, use_floor,
  stiffness_collision, stiffness_dirichlet, nonlinear_iter_count, pcg_iter_count, contact_energy_type) and
  the ``shells`` list -- model_name, translation, rotation (radians), scale, shell_type / material (Cloth or
  Rigid), fixed_points (method, range, fixed_info with rotation, translation and scale animations).
  Placement follows make_model_matrix = T * R * S with R = Rx Ry Rz as the reference writes them
  (Solver/Core/affine_position.h); pinned vertices follow set_pinned_verts_from_norm_position
  (Solver/Initializer/init_mesh_data.cpp:60-250): positions normalised by the model-space bounding box.

Edges, bending stencils, areas, masses, contact offsets and affine bodies are then derived by
``scenes.assemble`` exactly as for the synthetic scenes.

* ``save_state`` / ``load_state``: the frame state files of SolverInterface
  (Solver/SimulationSolver/solver_interface.cpp:206-412); ``write_obj``: the frame's meshes as
  ``save_mesh_to_obj`` writes them (:413-485).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import scenes as S


def read_obj(path):
    """(positions (n, 3) float32, faces (m, 3) uint32) of an OBJ file."""
    verts, faces = [], []
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "v" and len(tok) >= 4:
                verts.append((float(tok[1]), float(tok[2]), float(tok[3])))
            elif tok[0] == "f" and len(tok) >= 4:
                idx = []
                for t in tok[1:]:
                    k = int(t.split("/")[0])
                    idx.append(k - 1 if k > 0 else len(verts) + k)  # negative: relative to the end
                for i in range(1, len(idx) - 1):  # fan triangulation
                    a, b, c = idx[0], idx[i], idx[i + 1]
                    if a != b and a != c and b != c:
                        faces.append((a, b, c))
    x = np.asarray(verts, np.float32).reshape(-1, 3)
    f = np.asarray(faces, np.int64).reshape(-1, 3)
    if len(f) and (f.min() < 0 or f.max() >= len(x)):
        raise ValueError(f"{path}: face index out of range")
    return x, f.astype(np.uint32)


def _rot_x(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[1, 0, 0], [0, c, s], [0, -s, c]], np.float64)


def _rot_y(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, 0, -s], [0, 1, 0], [s, 0, c]], np.float64)


def _rot_z(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], np.float64)


def model_matrix(translation, rotation, scale):
    """make_model_matrix(t, r, s) = translate(t) * rotate(r) * scale(s) as a 3 x 4 affine map."""
    R = _rot_x(rotation[0]) @ _rot_y(rotation[1]) @ _rot_z(rotation[2])
    M = R @ np.diag(np.asarray(scale, np.float64))
    return M, np.asarray(translation, np.float64)


_SIDES = {
    "Left": lambda n, r: n[:, 0] < r, "Right": lambda n, r: n[:, 0] > 1 - r,
    "Front": lambda n, r: n[:, 2] < r, "Back": lambda n, r: n[:, 2] > 1 - r,
    "Up": lambda n, r: n[:, 1] > 1 - r, "Down": lambda n, r: n[:, 1] < r,
}
_COMBOS = {
    "LeftUp": ("Left", "Up"), "LeftDown": ("Left", "Down"), "RightUp": ("Right", "Up"),
    "RightDown": ("Right", "Down"), "FrontUp": ("Front", "Up"), "FrontDown": ("Front", "Down"),
    "BackUp": ("Back", "Up"), "BackDown": ("Back", "Down"),
}


def fixed_mask(model_x, method, rng=0.001):
    """Pinned vertices of a fixed_points entry (WorldData::load_fixed_points, init_mesh_data.cpp:116-250)."""
    lo, hi = model_x.min(0), model_x.max(0)
    n = (model_x - lo) * (np.float32(1.0) / np.maximum(hi - lo, np.float32(1e-4)))
    if method == "All":
        return np.ones(len(model_x), bool)
    if method == "None":
        return np.zeros(len(model_x), bool)
    if method in _SIDES:
        return _SIDES[method](n, rng)
    if method in _COMBOS:
        a, b = _COMBOS[method]
        return _SIDES[a](n, rng) & _SIDES[b](n, rng)
    if method == "LeftFront":  # the reference pairs Left with z > 1 - r ...
        return (n[:, 0] < rng) & (n[:, 2] > 1 - rng)
    if method == "LeftBack":   # ... and Back with z < r for the x-sided corners
        return (n[:, 0] < rng) & (n[:, 2] < rng)
    if method == "RightFront":
        return (n[:, 0] > 1 - rng) & (n[:, 2] > 1 - rng)
    if method == "RightBack":
        return (n[:, 0] > 1 - rng) & (n[:, 2] < rng)
    raise ValueError(f"fixed_points method {method!r} is not expressible in a scene file")


def _vec(v, default):
    return [float(a) for a in v[:3]] if isinstance(v, list) and len(v) >= 3 else list(default)


def _resolve(name, mesh_dirs):
    if os.path.isabs(name) and os.path.exists(name):
        return name
    for d in mesh_dirs:
        for cand in (os.path.join(d, name), os.path.join(d, os.path.basename(name))):
            if os.path.exists(cand):
                return cand
    raise FileNotFoundError(f"mesh {name!r} not found in {list(mesh_dirs)}")


def load_scene_json(path, mesh_dirs=()):
    """(Scene, solver settings) of a reference scene file.  mesh_dirs: folders searched for model_name
    (the reference's InputMesh folder).  Settings: dt, nonlinear_iters, pcg_max_iter, use_floor, floor_y,
    dirichlet -- the keyword arguments NewtonSolver takes."""
    with open(path) as fh:
        cfg = json.load(fh)
    if int(cfg.get("contact_energy_type", 1)) != 1:
        raise ValueError("only the barrier contact energy (contact_energy_type 1) is on this path")
    dt = float(cfg.get("implicit_dt", 1.0 / 60.0))
    gravity = _vec(cfg.get("gravity"), (0.0, -9.8, 0.0))
    kappa = float(cfg.get("stiffness_collision", 1e7))
    parts, anims_local, cloth_mats = [], [], []
    for shell in cfg.get("shells", []):
        name = shell.get("model_name", "")
        mx, mf = read_obj(_resolve(name, mesh_dirs))
        sc_ = shell.get("scale", 1.0)
        scale = [float(sc_)] * 3 if isinstance(sc_, (int, float)) else _vec(sc_, (1, 1, 1))
        M, t = model_matrix(_vec(shell.get("translation"), (0, 0, 0)), _vec(shell.get("rotation"), (0, 0, 0)), scale)
        x = (mx.astype(np.float64) @ M.T + t).astype(np.float32)
        mat = shell.get("material", {}) if isinstance(shell.get("material"), dict) else {}
        kind = mat.get("type", shell.get("shell_type", "Cloth"))
        if kind in ("Tetrahedral", "Tet", "TetMaterial", "Rod"):
            raise ValueError(f"shell type {kind!r} (tetrahedral / rod materials) is not on this path")
        if kind not in ("Cloth", "Rigid"):  # any other type string: a default cloth with thickness and d_hat only
            mat = {k: v for k, v in mat.items() if k in ("thickness", "d_hat")}
            kind = "Cloth"
        if kind == "Rigid" and mat.get("is_shell", True) is False:
            raise ValueError("solid rigid bodies (is_shell false) are not on this path")
        rigid = kind == "Rigid"
        thickness = float(mat.get("thickness", 2e-3))
        part = S.MeshPart(x, mf, np.zeros(len(x), bool), thickness=thickness, d_hat=float(mat.get("d_hat", 2e-3)),
                          density=float(mat.get("density", 1e3)), material_thickness=thickness, rigid=rigid,
                          rigid_stiffness=float(mat.get("stiffness", 1e6)))
        if float(mat.get("mass", 0.0)) != 0.0:
            part.total_mass = float(mat["mass"])
        if not rigid:
            part.youngs_modulus = float(mat.get("youngs_modulus", 1e5))
            part.poisson_ratio = float(mat.get("poisson_ratio", 0.25))
            part.area_bending_stiffness = float(mat.get("area_bending_stiffness", 5e-3))
            cloth_mats.append((_model(mat.get("stretch_model", 1)), _model(mat.get("bending_model", 2), bending=True)))
        for fp in shell.get("fixed_points", []):
            method = fp.get("method", "All")
            rng = fp.get("range", [0.001])
            sel = fixed_mask(mx, method, float(rng[0]) if rng else 0.001)
            part.pinned = part.pinned | sel
            fi = fp.get("fixed_info", {}) or {}
            mode = (1 if fi.get("use_rotate") else 0) | (2 if fi.get("use_scale") or "scale" in fi else 0) | \
                (4 if fi.get("use_translate") else 0)
            if mode and sel.any():
                anims_local.append((len(parts), np.nonzero(sel)[0], np.asarray(_vec(fi.get("rotCenter"), (0, 0, 0))),
                                    np.asarray(_vec(fi.get("rotAxis"), (1, 0, 0))),
                                    math.radians(float(fi.get("rotAngVelDeg", 0.0))),
                                    np.asarray(_vec(fi.get("translate"), (0, 0, 0))),
                                    np.asarray(_vec(fi.get("scale"), (1, 1, 1))), mode))
        parts.append(part)
    if len(set(cloth_mats)) > 1:
        raise ValueError("cloth shells with different stretch / bending models: one model per scene on this path")
    sm, bm = cloth_mats[0] if cloth_mats else (1, 2)
    sc = S.assemble(os.path.splitext(os.path.basename(path))[0], parts, dt=dt, gravity=gravity, kappa=kappa,
                    stretch_model=sm, bending_model=bm)
    sc.dirichlet = float(cfg.get("stiffness_dirichlet", 1e9))
    offs = np.cumsum([0] + [p.x.shape[0] for p in parts])
    sc.anims = [(vids + offs[m], c, a, w, tr, s, mode) for m, vids, c, a, w, tr, s, mode in anims_local]
    settings = dict(nonlinear_iters=int(cfg.get("nonlinear_iter_count", 3)),
                    pcg_max_iter=int(cfg.get("pcg_iter_count", 100)),
                    use_floor=bool(cfg.get("use_floor", True)), floor_y=0.0)
    return sc, settings


def _model(v, bending=False):
    names = ({"None": 0, "QuadraticBending": 1, "DihedralAngle": 2} if bending else {"Spring": 0, "FEM_BW98": 1})
    if isinstance(v, str):
        return names.get(v, 2 if bending else 1)
    return int(v)


def _mesh_verts(sc):
    return sc.num_verts - 4 * sc.num_bodies


def save_state(path, sc, x, v):
    """A frame state file as SolverInterface::save_current_frame_state_to_host writes it
    (solver_interface.cpp:206-273): sections ``o position`` and ``o velocity`` (one ``v x y z`` line per mesh
    vertex) and ``o q`` and ``o qv`` (four lines per affine body: p, a0, a1, a2 and their velocities).
    Values are written with 9 significant digits, so a float32 state reads back bit for bit."""
    V, NB = _mesh_verts(sc), sc.num_bodies
    x, v = np.asarray(x, np.float32), np.asarray(v, np.float32)
    slots = np.concatenate([np.arange(int(d), int(d) + 4) for d in sc.body_dof]) if NB else np.zeros(0, np.int64)

    def block(a):
        return "".join(f"v {r[0]:.9g} {r[1]:.9g} {r[2]:.9g}\n" for r in a[:, :3].tolist())
    with open(path, "w") as fh:
        fh.write("o position\n" + block(x[:V]) + "o velocity\n" + block(v[:V]) +
                 "o q\n" + block(x[slots]) + "o qv\n" + block(v[slots]))


def load_state(path, sc, like=None):
    """(positions, velocities) float32 (V, 4) of the scene from a frame state file
    (SolverInterface::load_saved_state_from_host, solver_interface.cpp:275-412).  ``like`` supplies the
    fourth lane (and is the starting copy); the body q and q velocities of the ``o q`` / ``o qv`` sections go
    to the bodies' DOF slots.  A section with more or fewer lines than the scene has vertices (bodies x 4)
    raises ValueError; a missing file raises FileNotFoundError."""
    V, NB = _mesh_verts(sc), sc.num_bodies
    sec = {"position": [], "velocity": [], "q": [], "qv": []}
    cur = None
    with open(path) as fh:
        for line in fh:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "o":
                cur = tok[1] if len(tok) > 1 and tok[1] in sec else None
                continue
            if tok[0] == "v" and cur is not None:
                sec[cur].append((float(tok[1]), float(tok[2]), float(tok[3])))
    want = {"position": V, "velocity": V, "q": 4 * NB, "qv": 4 * NB}
    for k, n in want.items():
        if len(sec[k]) != n:
            raise ValueError(f"{path}: section {k!r} holds {len(sec[k])} vertices, the scene has {n}")
    x = np.zeros((sc.num_verts, 4), np.float32) if like is None else np.array(like, np.float32, copy=True)
    v = np.zeros((sc.num_verts, 4), np.float32)
    x[:V, :3] = np.asarray(sec["position"], np.float32).reshape(-1, 3)
    v[:V, :3] = np.asarray(sec["velocity"], np.float32).reshape(-1, 3)
    if NB:
        slots = np.concatenate([np.arange(int(d), int(d) + 4) for d in sc.body_dof])
        x[slots, :3] = np.asarray(sec["q"], np.float32).reshape(-1, 3)
        v[slots, :3] = np.asarray(sec["qv"], np.float32).reshape(-1, 3)
    return x, v


def write_obj(path, sc, x):
    """The frame's meshes as SolverInterface::save_mesh_to_obj writes them (solver_interface.cpp:413-485):
    one ``o mesh_<k>`` object per mesh part with its vertices, faces indexed 1-based over the whole file."""
    x = np.asarray(x, np.float32)
    pv = sc.part_verts if sc.part_verts is not None else np.array([0, _mesh_verts(sc)])
    pf = sc.part_faces if sc.part_faces is not None else np.array([0, sc.faces.shape[0]])
    out = ["# simulated result\n"]
    for k in range(len(pv) - 1):
        out.append(f"o mesh_{k}\n")
        out.extend(f"v {r[0]:.9g} {r[1]:.9g} {r[2]:.9g}\n" for r in x[pv[k]:pv[k + 1], :3].tolist())
        out.extend(f"f {a + 1} {b + 1} {c + 1}\n" for a, b, c in sc.faces[pf[k]:pf[k + 1], :3].tolist())
    with open(path, "w") as fh:
        fh.write("".join(out))
