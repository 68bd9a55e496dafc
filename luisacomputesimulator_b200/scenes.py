"""Seeded synthetic scenes with the shapes of the reference's benchmark configurations.

No mesh file or dataset is read: the cloth grids, the icosphere and the twisted tube are
generated here, and the per-element data the contact path consumes is derived the way the
reference's initialisers derive it:

* edges: unique (min, max) vertex pairs in lexicographic order, the order
  ``extract_edges_from_surface`` produces (Solver/MeshOperation/mesh_reader.cpp:219-300);
* dihedral (bending) stencils ``(e0, e1, opposite-of-first-face, opposite-of-second-face)``
  for every interior edge (mesh_reader.cpp:219-300);
* rest areas: face area, vertex area = sum(adjacent face area / 3) in double, edge area =
  sum(adjacent face area / 3) (Solver/Initializer/init_mesh_data.cpp:780-870);
* contact offset and d_hat per vertex, scaled down when offset + d_hat reaches 0.9 x the
  smallest rest edge length / triangle altitude of the mesh
  (Solver/Initializer/init_collision_data.cpp:67-171);
* pinned vertices and their animated targets (Solver/Initializer/init_mesh_data.cpp:116-170,
  Solver/SimulationSolver/solver_interface.cpp:130-162);
* the cloth material of ClothMaterial's defaults (Solver/SimulationCore/physical_material.h:53-62):
  Baraff-Witkin stretch faces with rest Dm^-1 (StretchEnergy::get_Dm_inv, Solver/Energy/stretch_energy.h:424-438),
  rest area and mu = lambda = E / (2 (1 + nu)) resp. E nu / ((1 + nu)(1 - 2 nu)) scaled by the thickness
  (E = 1e5, nu = 0.25, thickness 2e-3: 80 each; Solver/Initializer/init_sim_data.cpp:370-397), and
  dihedral bending with the rest angle and h_bar = (A0 + A1) / (3 |e|) per stencil
  (init_sim_data.cpp:400-448).  Elements whose vertices are all pinned are dropped
  (init_sim_data.cpp:205-270).  The material thickness only scales the stiffnesses; the contact
  thickness of a mesh part is separate (0 in the benchmark configurations).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class MeshPart:
    x: np.ndarray          # (n, 3) float32
    faces: np.ndarray      # (f, 3) uint32, local indices
    pinned: np.ndarray     # (n,) bool
    thickness: float = 0.0
    d_hat: float = 1e-3
    density: float = 1e3   # kg / m^3 (MaterialBase::density)
    material_thickness: float = 2e-3  # ClothMaterial::thickness: shell volume = area x thickness
    rotate: tuple | None = None  # pinned-vertex animation: (axis_point(3), axis(3), ang_vel, mask)
    rigid: bool = False    # an affine body (RigidMaterial): 12 DOFs q = [p, a0, a1, a2], x = p + A x_bar
    rigid_stiffness: float = 1e6  # RigidMaterial::stiffness (orthogonality kappa)
    total_mass: float | None = None  # MaterialBase::mass: the part's mass when given (else volume x density)
    youngs_modulus: float | None = None      # ClothMaterial (None: the scene's lame_params)
    poisson_ratio: float | None = None
    area_bending_stiffness: float | None = None


@dataclasses.dataclass
class Scene:
    name: str
    x: np.ndarray            # (V, 4) float32 rest / initial positions
    faces: np.ndarray        # (F, 4) uint32
    edges: np.ndarray        # (E, 2) uint32
    bending: np.ndarray      # (B, 4) uint32
    vert_area: np.ndarray    # (V,) float32
    face_area: np.ndarray    # (F,) float32
    edge_area: np.ndarray    # (E,) float32
    mass: np.ndarray         # (V,) float32
    pinned: np.ndarray       # (V,) uint8
    d_hat: np.ndarray        # (V,) float32
    offset: np.ndarray       # (V,) float32
    body: np.ndarray         # (V,) uint32, 0xFFFFFFFF = soft
    rest_len: np.ndarray     # (E,) float32
    bending_Q: np.ndarray    # (B, 4, 4) float32
    dt: float = 1.0 / 60.0
    gravity: tuple = (0.0, -9.8, 0.0)
    kappa: float = 1e7
    spring_k: float = 1e4
    bending_k: float = 5e-3
    dirichlet: float = 1e9
    anims: list = dataclasses.field(default_factory=list)  # (vertex ids, center, axis, omega)
    # cloth material (ConstitutiveStretchModelCloth / ConstitutiveBendingModelCloth values)
    stretch_model: int = 1                # 0 spring, 1 BW98
    bending_model: int = 2                # 0 none, 1 quadratic, 2 dihedral
    stretch_faces: np.ndarray = None      # (Fs, 4) uint32
    stretch_dm_inv: np.ndarray = None     # (Fs, 4) float32: rest Dm^-1 columns
    stretch_area: np.ndarray = None       # (Fs,) float32
    stretch_mu: float = 80.0
    stretch_lambda: float = 80.0
    bending_rest_angle: np.ndarray = None  # (B,) float32
    bending_hbar: np.ndarray = None        # (B,) float32
    bending_scaling: float = 1.0           # stiffness_bending_ui
    # affine bodies: the 4 DOF slots of body b are vertices body_dof[b] .. body_dof[b] + 3 holding
    # p, a0, a1, a2 (not part of any face, edge or contact query: d_hat < 0); rigid vertices carry
    # their body id in `body` and their body-frame position in model_x
    body_dof: np.ndarray = None            # (NB,) uint32
    body_mass: np.ndarray = None           # (NB, 4, 4) float32: [M, MI^T; MI, I] (init_sim_data.cpp:640-703)
    body_volume: np.ndarray = None         # (NB,) float32
    body_kappa: np.ndarray = None          # (NB,) float32
    model_x: np.ndarray = None             # (V, 4) float32
    # per-element material parameters (one value per scene unless the parts' materials differ)
    stretch_mu_lambda: np.ndarray = None   # (Fs, 2) float32
    bending_stiffness: np.ndarray = None   # (B,) float32
    spring_stiffness: np.ndarray = None    # (E,) float32
    # mesh parts in order: vertex and face offsets (num_parts + 1 each; the DOF slots follow the last part)
    part_verts: np.ndarray = None
    part_faces: np.ndarray = None

    @property
    def num_bodies(self):
        return 0 if self.body_dof is None else int(self.body_dof.shape[0])

    @property
    def num_verts(self):
        return self.x.shape[0]

    def targets(self, t):
        """Positions of the pinned vertices at time t (others: rest position): scale, rotation, translation
        (FixedPointAnimationInfo::fn_affine_position, init_mesh_data.h:61-92)."""
        out = self.x[:, :3].astype(np.float64).copy()
        for an in self.anims:
            vids, center, axis, omega = an[:4]
            translate, scale, mode = (an[4], an[5], an[6]) if len(an) > 4 else (None, None, 1)
            p = out[vids]
            if mode & 2:
                p = np.asarray(scale, np.float64) * t * p
            if mode & 1:
                p = _rotate(p - center, axis, omega * t) + center
            if mode & 4:
                p = p + np.asarray(translate, np.float64) * t
            out[vids] = p
        return out.astype(np.float32)


def scaled_offset_d_hat(thickness, d_hat, min_rest_dist, rigid):
    """Contact offset and d_hat of one mesh (init_collision_data.cpp:106-146, in float32 as there): offset =
    thickness / 2; when offset + d_hat reaches the safe distance 0.9 x the mesh's smallest rest edge length /
    triangle altitude, the offset is cut to half the safe distance and d_hat to what is left.  A rigid body's
    safe distance is 1e8, which exempts it."""
    f = np.float32
    safe = f(1e8) if rigid else f(0.9) * f(min_rest_dist)
    so, sd = f(0.5) * f(thickness), f(d_hat)
    if not (so + sd < safe):
        if so > f(0.5) * safe:
            so = f(0.5) * safe
        if sd > safe - so:
            sd = safe - so
    return float(so), float(sd)


def _rotate(p, axis, ang):
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    c, s = math.cos(ang), math.sin(ang)
    return p * c + np.cross(axis, p) * s + np.outer(p @ axis, axis) * (1 - c)


def cloth_grid(nx, nz, spacing, origin=(0.0, 0.0, 0.0), jitter=1e-4, seed=0):
    """nx x nz vertex grid in the x-z plane, row-major, each quad split on its (i,j)-(i+1,j+1)
    diagonal; out-of-plane (y) jitter U(-jitter, jitter)."""
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    x = np.zeros((nx * nz, 3), np.float64)
    x[:, 0] = origin[0] + (ii.ravel() - (nx - 1) / 2.0) * spacing
    x[:, 2] = origin[2] + (jj.ravel() - (nz - 1) / 2.0) * spacing
    x[:, 1] = origin[1] + rng.uniform(-jitter, jitter, nx * nz)
    vid = lambda i, j: i * nz + j  # noqa: E731
    faces = []
    for i in range(nx - 1):
        for j in range(nz - 1):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            faces.append((a, b, c))
            faces.append((a, c, d))
    return x.astype(np.float32), np.asarray(faces, np.uint32)


def icosphere(subdiv, radius, center=(0.0, 0.0, 0.0)):
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.asarray(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    x = np.asarray(verts) * radius + np.asarray(center)
    return x.astype(np.float32), np.asarray(faces, np.uint32)


def tube(n_around, n_along, radius, length, center=(0.0, 0.0, 0.0)):
    """Periodic cylinder around the x axis: n_around x n_along grid, vertex (i around, j along)
    at index j * n_around + i; quads split on their (i,j)-(i+1,j+1) diagonal."""
    th = 2.0 * np.pi * np.arange(n_around) / n_around
    xs = -length / 2.0 + length * np.arange(n_along) / (n_along - 1)
    J, I = np.meshgrid(np.arange(n_along), np.arange(n_around), indexing="ij")
    x = np.zeros((n_along * n_around, 3), np.float64)
    x[:, 0] = center[0] + xs[J.ravel()]
    x[:, 1] = center[1] + radius * np.cos(th[I.ravel()])
    x[:, 2] = center[2] + radius * np.sin(th[I.ravel()])
    vid = lambda i, j: j * n_around + (i % n_around)  # noqa: E731
    faces = []
    for j in range(n_along - 1):
        for i in range(n_around):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            faces.append((a, b, c))
            faces.append((a, c, d))
    return x.astype(np.float32), np.asarray(faces, np.uint32)


def box_mesh(size, center):
    """Closed box surface (8 vertices, 12 triangles)."""
    h = np.asarray(size, np.float64) / 2.0
    c = np.asarray(center, np.float64)
    x = np.asarray([[sx, sy, sz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], np.float64) * h + c
    f = [(0, 1, 3), (0, 3, 2), (4, 6, 7), (4, 7, 5), (0, 4, 5), (0, 5, 1), (2, 3, 7), (2, 7, 6), (0, 2, 6),
         (0, 6, 4), (1, 5, 7), (1, 7, 3)]
    return x.astype(np.float32), np.asarray(f, np.uint32)


def extract_edges(faces):
    """Unique sorted edges and dihedral stencils (mesh_reader.cpp:219-300 ordering)."""
    f = np.sort(faces.astype(np.int64), axis=1)
    nf = f.shape[0]
    fid = np.arange(nf)
    half = np.concatenate([np.stack([f[:, 0], f[:, 1], fid], 1), np.stack([f[:, 0], f[:, 2], fid], 1),
                           np.stack([f[:, 1], f[:, 2], fid], 1)])
    order = np.lexsort((half[:, 2], half[:, 1], half[:, 0]))
    half = half[order]
    same_next = np.zeros(len(half), bool)
    same_next[:-1] = (half[1:, 0] == half[:-1, 0]) & (half[1:, 1] == half[:-1, 1])
    same_prev = np.zeros(len(half), bool)
    same_prev[1:] = same_next[:-1]
    keep = ~same_next  # types 0 (boundary) and 2 (second of an interior pair)
    edges = half[keep][:, :2].astype(np.uint32)
    # dihedral stencils from interior pairs (first element of each pair)
    firsts = np.nonzero(same_next)[0]
    bend = []
    fa = faces.astype(np.int64)
    for k in firsts:
        a, b, f1 = half[k]
        f2 = half[k + 1, 2]
        o1 = [v for v in fa[f1] if v != a and v != b][0]
        o2 = [v for v in fa[f2] if v != a and v != b][0]
        bend.append((a, b, o1, o2))
    bending = np.asarray(bend, np.uint32).reshape(-1, 4)
    # adjacency edge -> faces for edge areas
    edge_faces = np.full((edges.shape[0], 2), -1, np.int64)
    eidx = np.cumsum(keep) - 1  # index of the edge each half belongs to (pairs share the later one)
    eidx_first = np.where(same_next, eidx + 1, eidx)
    for k in range(len(half)):
        e = eidx_first[k]
        slot = 0 if edge_faces[e, 0] < 0 else 1
        edge_faces[e, slot] = half[k, 2]
    return edges, bending, edge_faces


def _face_area(x, faces):
    x = x.astype(np.float32)
    v0 = x[faces[:, 1]] - x[faces[:, 0]]
    v1 = x[faces[:, 2]] - x[faces[:, 0]]
    return (np.linalg.norm(np.cross(v0, v1), axis=1) * np.float32(0.5)).astype(np.float32)


def _bending_Q(x, bend):
    """Q = 3/(A0+A1) K K^T of the quadratic bending model (init_sim_data.cpp:455-480)."""
    x = x.astype(np.float64)
    p = [x[bend[:, k]] for k in range(4)]
    e0, e1, e2, e3, e4 = p[1] - p[0], p[2] - p[0], p[3] - p[0], p[2] - p[1], p[3] - p[1]

    def cot(a, b):
        return np.einsum("ij,ij->i", a, b) / np.linalg.norm(np.cross(a, b), axis=1)

    c01, c02, c03, c04 = cot(e0, -e1), cot(e0, -e2), cot(e0, e3), cot(e0, e4)
    K = np.stack([c03 + c04, c01 + c02, -c01 - c03, -c02 - c04], 1)
    A0 = 0.5 * np.linalg.norm(np.cross(e0, e1), axis=1)
    A1 = 0.5 * np.linalg.norm(np.cross(e0, e2), axis=1)
    Q = (3.0 / (A0 + A1))[:, None, None] * K[:, :, None] * K[:, None, :]
    return Q.astype(np.float32)


def lame(youngs_modulus=1e5, poisson_ratio=0.25, thickness=2e-3):
    """StretchEnergy::convert_prop (stretch_energy.h:418-423) scaled by the thickness, as float32."""
    mu = youngs_modulus / (2.0 * (1.0 + poisson_ratio))
    lam = youngs_modulus * poisson_ratio / ((1.0 + poisson_ratio) * (1.0 - 2.0 * poisson_ratio))
    return float(np.float32(np.float32(thickness) * mu)), float(np.float32(np.float32(thickness) * lam))


def _dm_inv(x, faces):
    """StretchEnergy::get_Dm_inv per face: the 2D rest edge matrix in the triangle's own frame,
    inverted; 4 floats per face = its columns."""
    x = x.astype(np.float64)
    x0, x1, x2 = x[faces[:, 0]], x[faces[:, 1]], x[faces[:, 2]]
    r1, r2 = x1 - x0, x2 - x0
    n = np.cross(r1, r2)
    a1 = r1 / np.linalg.norm(r1, axis=1)[:, None]
    a2 = np.cross(n, a1)
    a2 = a2 / np.linalg.norm(a2, axis=1)[:, None]
    uv = [np.stack([np.einsum("ij,ij->i", a1, p), np.einsum("ij,ij->i", a2, p)], 1) for p in (x0, x1, x2)]
    d0, d1 = uv[1] - uv[0], uv[2] - uv[0]          # columns of Dm
    a, b, c, d = d0[:, 0], d0[:, 1], d1[:, 0], d1[:, 1]
    det = a * d - c * b
    return np.stack([d / det, -b / det, -c / det, a / det], 1).astype(np.float32)


def dihedral_angle(p0, p1, p2, p3):
    """Signed dihedral angle of hinge (p0, p1) with wings p2, p3 (face_dihedral_angle(p2, p1, p0, p3),
    bending_energy.h:222-231), float32."""
    f = np.float32
    n1 = np.cross(p1 - p2, p0 - p2).astype(f)
    n2 = np.cross(p0 - p3, p1 - p3).astype(f)
    c = np.einsum("ij,ij->i", n1, n2) / np.sqrt(np.einsum("ij,ij->i", n1, n1) * np.einsum("ij,ij->i", n2, n2))
    ang = np.arccos(np.clip(c, f(-1), f(1))).astype(f)
    return (np.sign(np.einsum("ij,ij->i", np.cross(n2, n1), p1 - p0)) * ang).astype(f)


def _dihedral_rest(x, bend):
    """Rest angle and h_bar = (A0 + A1) / (3 |e|) per stencil (init_sim_data.cpp:420-436)."""
    x = x.astype(np.float32)
    p = [x[bend[:, k]] for k in range(4)]
    ang = dihedral_angle(*p)
    a0 = np.linalg.norm(np.cross(p[1] - p[0], p[2] - p[0]), axis=1) * np.float32(0.5)
    a1 = np.linalg.norm(np.cross(p[1] - p[0], p[3] - p[0]), axis=1) * np.float32(0.5)
    l0 = np.linalg.norm(p[0] - p[1], axis=1)
    return ang.astype(np.float32), ((a0 + a1) / (np.float32(3.0) * l0)).astype(np.float32)


def _min_rest_dist(x, faces, edges):
    x = x.astype(np.float32)
    lens = np.linalg.norm(x[edges[:, 0]] - x[edges[:, 1]], axis=1)
    best = float(lens.min()) if len(lens) else 1e10
    for k in range(3):
        v0, v1, v2 = x[faces[:, k]], x[faces[:, (k + 1) % 3]], x[faces[:, (k + 2) % 3]]
        r = v2 - v1
        d = np.einsum("ij,ij->i", r, r)
        t = np.where(d > 1.19209290e-7, np.einsum("ij,ij->i", r, v0 - v1) / np.maximum(d, 1e-30), 0.5)
        cp = (1 - t)[:, None] * v1 + t[:, None] * v2
        best = min(best, float(np.linalg.norm(cp - v0, axis=1).min()))
    return best


def assemble(name, parts, dt, gravity, kappa, spring_k=None, bending_k=5e-3, stretch_model=1, bending_model=2,
             lame_params=(1e5, 0.25, 2e-3)):
    """Merge mesh parts into one Scene (vertex/face order = part order; the DOF slots of rigid parts,
    four per body, follow all mesh vertices)."""
    xs, fs, pins, vmesh, anims = [], [], [], [], []
    off = 0
    for m, part in enumerate(parts):
        xs.append(part.x)
        fs.append(part.faces.astype(np.int64) + off)
        pins.append(part.pinned)
        vmesh.append(np.full(part.x.shape[0], m))
        if part.rotate is not None:
            center, axis, omega, mask = part.rotate
            anims.append((np.nonzero(mask)[0] + off, np.asarray(center), np.asarray(axis), float(omega)))
        off += part.x.shape[0]
    x3 = np.concatenate(xs).astype(np.float32)
    faces = np.concatenate(fs).astype(np.uint32)
    edges, bending, edge_faces = extract_edges(faces)
    face_area = _face_area(x3, faces)
    V = x3.shape[0]
    vert_area = np.zeros(V, np.float64)
    for k in range(3):
        np.add.at(vert_area, faces[:, k], face_area.astype(np.float64) / 3.0)
    ef = edge_faces
    edge_area = np.where(ef[:, 0] >= 0, face_area[np.maximum(ef[:, 0], 0)] / 3.0, 0.0) + \
        np.where(ef[:, 1] >= 0, face_area[np.maximum(ef[:, 1], 0)] / 3.0, 0.0)
    vmesh = np.concatenate(vmesh)
    d_hat = np.zeros(V, np.float32)
    offset = np.zeros(V, np.float32)
    mass = np.zeros(V, np.float32)
    foff = 0
    for m, part in enumerate(parts):
        nfm = part.faces.shape[0]
        sel_f = slice(foff, foff + nfm)
        foff += nfm
        vm = vmesh == m
        fe = faces[sel_f]
        emask = vm[edges[:, 0]]
        so, sd = scaled_offset_d_hat(part.thickness, part.d_hat, _min_rest_dist(x3, fe, edges[emask]), part.rigid)
        d_hat[vm] = sd
        offset[vm] = so
        # vertex mass = vertex volume / body volume x body mass, shell volumes = area x thickness
        # (init_mesh_data.cpp:826-845, 884-898, 946-990)
        th = np.float32(part.material_thickness)
        vert_vol = (vert_area[vm] * th).astype(np.float32)
        body_vol = float(np.sum(face_area[sel_f].astype(np.float64) * th))
        body_mass = np.float32(part.total_mass if part.total_mass else body_vol * part.density)
        mass[vm] = (vert_vol / np.float32(body_vol) * body_mass).astype(np.float32)
    x4 = np.zeros((V, 4), np.float32)
    x4[:, :3] = x3
    f4 = np.zeros((faces.shape[0], 4), np.uint32)
    f4[:, :3] = faces
    body = np.full(V, 0xFFFFFFFF, np.uint32)
    rest_len = np.linalg.norm(x3[edges[:, 0]] - x3[edges[:, 1]], axis=1).astype(np.float32)
    pinned = np.concatenate(pins).astype(np.uint8)
    # cloth elements: of cloth parts, with a free vertex (init_sim_data.cpp:205-270)
    rigid_v = np.zeros(V, bool)
    for m, part in enumerate(parts):
        if part.rigid:
            rigid_v[vmesh == m] = True
    free = (pinned == 0) & ~rigid_v
    bending = bending[free[bending].any(axis=1) & ~rigid_v[bending].any(axis=1)] if len(bending) else bending
    sf = faces[free[faces].any(axis=1) & ~rigid_v[faces].any(axis=1)]
    # affine bodies (init_sim_data.cpp:520-757): q = [p, a0, a1, a2] with p the part's centroid and A = I
    # at rest, x_bar = x - p; mass matrix from the vertex masses, diagonal clamped to >= Epsilon; volume
    # = area x thickness (shell); four DOF slots appended per body
    rig = [m for m, part in enumerate(parts) if part.rigid]
    NB = len(rig)
    model_x = np.zeros((V + 4 * NB, 4), np.float32)
    body_dof = np.zeros(NB, np.uint32)
    body_mass = np.zeros((NB, 4, 4), np.float32)
    body_volume = np.zeros(NB, np.float32)
    body_kappa = np.zeros(NB, np.float32)
    slot_x = np.zeros((4 * NB, 3), np.float32)
    foff_m = np.concatenate([[0], np.cumsum([p.faces.shape[0] for p in parts])])
    for b, m in enumerate(rig):
        vm = np.nonzero(vmesh == m)[0]
        body[vm] = b
        pc = x3[vm].astype(np.float64).mean(axis=0).astype(np.float32)
        xb = (x3[vm] - pc).astype(np.float32)
        model_x[vm, :3] = xb
        mv = mass[vm].astype(np.float64)
        Mb = mv.sum()
        MI = (mv[:, None] * xb).sum(0)
        Ib = (mv[:, None, None] * xb[:, :, None] * xb[:, None, :]).sum(0)
        Mm = np.zeros((4, 4))
        Mm[0, 0] = Mb
        Mm[0, 1:] = Mm[1:, 0] = MI
        Mm[1:, 1:] = Ib
        Mm[np.arange(4), np.arange(4)] = np.maximum(Mm[np.arange(4), np.arange(4)], 1.19209290e-7)
        body_mass[b] = Mm.astype(np.float32)
        body_volume[b] = np.float32(face_area[foff_m[m]:foff_m[m + 1]].astype(np.float64).sum() *
                                    parts[m].material_thickness)
        body_kappa[b] = parts[m].rigid_stiffness
        body_dof[b] = V + 4 * b
        slot_x[4 * b] = pc
        slot_x[4 * b + 1:4 * b + 4] = np.eye(3, dtype=np.float32)
    if NB:
        Vt = V + 4 * NB
        x3 = np.concatenate([x3, slot_x])
        x4 = np.zeros((Vt, 4), np.float32)
        x4[:, :3] = x3
        slot_body = np.repeat(np.arange(NB, dtype=np.uint32), 4)
        body = np.concatenate([body, slot_body])
        vert_area = np.concatenate([vert_area, np.zeros(4 * NB)])
        mass = np.concatenate([mass, np.zeros(4 * NB, np.float32)])
        pinned = np.concatenate([pinned, np.zeros(4 * NB, np.uint8)])
        d_hat = np.concatenate([d_hat, np.full(4 * NB, -1.0, np.float32)])  # no contact queries
        offset = np.concatenate([offset, np.zeros(4 * NB, np.float32)])
    sf4 = np.zeros((sf.shape[0], 4), np.uint32)
    sf4[:, :3] = sf
    mu, lam = lame(*lame_params)
    rest_angle, hbar = _dihedral_rest(x3, bending) if len(bending) else (np.zeros(0, np.float32),) * 2
    # per-element materials: each element takes its part's (mesh of its first vertex)
    part_ml = np.zeros((len(parts), 2), np.float32)
    part_kb = np.zeros(len(parts), np.float32)
    for m, part in enumerate(parts):
        E_, nu_, th_ = lame_params
        if part.youngs_modulus is not None:
            E_ = part.youngs_modulus
        if part.poisson_ratio is not None:
            nu_ = part.poisson_ratio
        part_ml[m] = lame(E_, nu_, part.material_thickness if part.youngs_modulus is not None else th_)
        part_kb[m] = bending_k if part.area_bending_stiffness is None else part.area_bending_stiffness
    vm_all = np.concatenate([vmesh, np.zeros(4 * NB, vmesh.dtype)]) if NB else vmesh
    stretch_ml = part_ml[vm_all[sf[:, 0]]] if len(sf) else np.zeros((0, 2), np.float32)
    bend_k = part_kb[vm_all[bending[:, 0]]] if len(bending) else np.zeros(0, np.float32)
    spring_k_e = part_ml[vm_all[edges[:, 0]], 0] if len(edges) else np.zeros(0, np.float32)
    return Scene(name=name, x=x4, faces=f4, edges=edges.astype(np.uint32), bending=bending.astype(np.uint32),
                 vert_area=vert_area.astype(np.float32), face_area=face_area, edge_area=edge_area.astype(np.float32),
                 mass=mass, pinned=pinned, d_hat=d_hat, offset=offset, body=body,
                 rest_len=rest_len, bending_Q=_bending_Q(x3, bending), dt=dt, gravity=tuple(gravity), kappa=kappa,
                 spring_k=mu if spring_k is None else spring_k, bending_k=bending_k, anims=anims,
                 stretch_model=stretch_model, bending_model=bending_model, stretch_faces=sf4,
                 stretch_dm_inv=_dm_inv(x3, sf), stretch_area=_face_area(x3, sf), stretch_mu=mu, stretch_lambda=lam,
                 bending_rest_angle=rest_angle, bending_hbar=hbar,
                 body_dof=body_dof if NB else None, body_mass=body_mass if NB else None,
                 body_volume=body_volume if NB else None, body_kappa=body_kappa if NB else None,
                 model_x=model_x if NB else None, stretch_mu_lambda=stretch_ml.astype(np.float32),
                 bending_stiffness=bend_k.astype(np.float32),
                 spring_stiffness=(spring_k_e if spring_k is None else np.full(len(edges), spring_k)).astype(np.float32),
                 part_verts=np.concatenate([[0], np.cumsum([p.x.shape[0] for p in parts])]).astype(np.int64),
                 part_faces=np.concatenate([[0], np.cumsum([p.faces.shape[0] for p in parts])]).astype(np.int64))


def cloth_on_sphere(n=64, spacing=0.01, seed=0, subdiv=4, radius=0.2, drop=0.05):
    """Config 1: n x n cloth (1 cm spacing) dropped from 5 cm above a pinned icosphere."""
    cx, cf = cloth_grid(n, n, spacing, origin=(0.0, radius + drop, 0.0), jitter=1e-4, seed=seed)
    sx, sf = icosphere(subdiv, radius)
    cloth = MeshPart(cx, cf, np.zeros(cx.shape[0], bool))
    sphere = MeshPart(sx, sf, np.ones(sx.shape[0], bool))
    return assemble(f"cloth{n}x{n}_on_sphere", [cloth, sphere], dt=1.0 / 60.0, gravity=(0, -9.8, 0), kappa=1e7)


def twisted_tube(n_around=300, n_along=296, radius=0.15, length=0.6, omega=2.0):
    """Config 2: periodic tube whose two end rings rotate at -+omega rad/s about the x axis."""
    x, f = tube(n_around, n_along, radius, length)
    V = x.shape[0]
    xn = (x[:, 0] - x[:, 0].min()) / (x[:, 0].max() - x[:, 0].min())
    left = xn < 0.001
    right = xn > 0.999
    part = MeshPart(x, f, left | right)
    sc = assemble(f"tube{n_around}x{n_along}", [part], dt=1.0 / 100.0, gravity=(0, 0, 0), kappa=1e9)
    sc.anims = [(np.nonzero(left)[0], np.zeros(3), np.array([1.0, 0, 0]), -omega),
                (np.nonzero(right)[0], np.zeros(3), np.array([1.0, 0, 0]), omega)]
    assert V == sc.num_verts
    return sc


def random_cloth_scene(n_verts, seed, collider="sphere"):
    """Batching/serving scenes: square cloth of ~n_verts over a seeded sphere or box collider."""
    side = max(4, int(round(math.sqrt(n_verts))))
    rng = np.random.default_rng(seed)
    spacing = 0.6 / side
    cx, cf = cloth_grid(side, side, spacing, origin=(0.0, 0.25, 0.0), jitter=1e-4, seed=seed)
    if collider == "sphere":
        sx, sf = icosphere(3, 0.2 * float(rng.uniform(0.8, 1.2)))
    else:
        sx, sf = box_mesh((0.3, 0.3, 0.3), (0.0, 0.0, 0.0))
    return assemble(f"cloth{side}_{collider}_{seed}",
                    [MeshPart(cx, cf, np.zeros(cx.shape[0], bool)), MeshPart(sx, sf, np.ones(sx.shape[0], bool))],
                    dt=1.0 / 60.0, gravity=(0, -9.8, 0), kappa=1e7)


def cloth_box_scene(n_verts, seed, box=0.08, gap=2e-3, collider=True):
    """A square cloth of ~n_verts over a seeded sphere (pinned) with an affine rigid box (8 vertices,
    12 DOFs, RigidMaterial) resting `gap` above the cloth's centre: the coupled scenes of the batching
    configuration."""
    side = max(4, int(round(math.sqrt(n_verts))))
    rng = np.random.default_rng(seed)
    spacing = 0.6 / side
    cy = 0.25
    cx, cf = cloth_grid(side, side, spacing, origin=(0.0, cy, 0.0), jitter=1e-4, seed=seed)
    parts = [MeshPart(cx, cf, np.zeros(cx.shape[0], bool))]
    if collider:
        sx, sf = icosphere(3, 0.2 * float(rng.uniform(0.8, 1.2)))
        parts.append(MeshPart(sx, sf, np.ones(sx.shape[0], bool)))
    bx, bf = box_mesh((box, box, box), (0.0, float(cx[:, 1].max()) + gap + box / 2.0, 0.0))
    parts.append(MeshPart(bx, bf, np.zeros(8, bool), rigid=True))
    return assemble(f"cloth{side}_box_{seed}", parts, dt=1.0 / 60.0, gravity=(0, -9.8, 0), kappa=1e7)
