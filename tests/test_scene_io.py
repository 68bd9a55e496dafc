"""Scene ingestion (luisacomputesimulator_b200/scene_io.py) on generated files: OBJ parsing, placement,
materials, rigid shells, fixed points and their animations; and, where the reference's resources are on
this machine, every scene file whose meshes ship with it."""
import glob
import json
import math
import os

import numpy as np
import pytest

from luisacomputesimulator_b200 import scene_io, scenes as S

# the reference's Resources folder, read only when REFERENCE_ROOT names the reference project's root
REF = os.path.join(os.environ["REFERENCE_ROOT"], "Resources") if os.environ.get("REFERENCE_ROOT") else ""


def _grid_obj(path, n=5, quads=True):
    lines = [f"v {i / (n - 1):.6f} 0 {j / (n - 1):.6f}" for i in range(n) for j in range(n)]
    for i in range(n - 1):
        for j in range(n - 1):
            a, b, c, d = i * n + j + 1, (i + 1) * n + j + 1, (i + 1) * n + j + 2, i * n + j + 2
            lines.append(f"f {a}/1/1 {b}/1/1 {c}/1/1 {d}/1/1" if quads else f"f {a} {b} {c}\nf {a} {c} {d}")
    open(path, "w").write("\n".join(lines) + "\n")


def test_read_obj_fans_polygons_and_drops_degenerate_faces(tmp_path):
    p = tmp_path / "m.obj"
    open(p, "w").write("# test\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\n"
                       "f 1/1/1 2/1/1 3/1/1 4/1/1\nf -4 -3 -3\nf 1//1 3//1 4//1\n")
    x, f = scene_io.read_obj(str(p))
    assert x.shape == (4, 3) and x.dtype == np.float32
    np.testing.assert_array_equal(f, [[0, 1, 2], [0, 2, 3], [0, 2, 3]])  # the quad fanned; (1, 2, 2) dropped


def test_scene_file_placement_materials_pins_and_animation(tmp_path):
    _grid_obj(tmp_path / "grid.obj")
    scene = {
        "implicit_dt": 0.02, "gravity": [0, -5, 0], "use_floor": False, "stiffness_collision": 3e6,
        "nonlinear_iter_count": 2, "pcg_iter_count": 40,
        "shells": [
            {"model_name": "grid.obj", "translation": [0, 1, 0], "scale": 2.0, "rotation": [0, 0, 0],
             "material": {"type": "Cloth", "youngs_modulus": 2e5, "poisson_ratio": 0.3,
                          "area_bending_stiffness": 0.1, "thickness": 1e-3},
             "fixed_points": [{"method": "Left", "range": [0.01],
                               "fixed_info": {"use_translate": True, "translate": [0, 1, 0]}},
                              {"method": "Right", "fixed_info": {"use_rotate": True, "rotCenter": [1, 1, 0],
                                                                 "rotAxis": [1, 0, 0], "rotAngVelDeg": 90}}]},
            {"model_name": "grid.obj", "translation": [0.5, 1.2, 0.5], "scale": [0.1, 0.1, 0.1],
             "rotation": [0, 0, math.pi / 2], "shell_type": "Rigid"},
        ]}
    p = tmp_path / "scene.json"
    p.write_text(json.dumps(scene))
    sc, st = scene_io.load_scene_json(str(p), [str(tmp_path)])
    assert st == dict(nonlinear_iters=2, pcg_max_iter=40, use_floor=False, floor_y=0.0)
    assert sc.dt == pytest.approx(0.02) and sc.gravity == (0, -5, 0) and sc.kappa == pytest.approx(3e6)
    # placement: scale 2 then translate; the rigid part rotated by the reference's Rz
    np.testing.assert_allclose(sc.x[:25, :3].min(0), [0, 1, 0], atol=1e-6)
    np.testing.assert_allclose(sc.x[:25, :3].max(0), [2, 1, 2], atol=1e-6)
    Rz = scene_io._rot_z(math.pi / 2)
    want = (np.asarray([[1.0, 0, 0]]) * 0.1) @ Rz.T + [0.5, 1.2, 0.5]
    np.testing.assert_allclose(sc.x[25 + 20, :3], want[0], atol=1e-6)  # model vertex (1, 0, 0) of the second part
    # pins: Left (x < 0.01 of the box) and Right (x > 0.999), five each
    assert sc.pinned[:25].sum() == 10
    assert len(sc.anims) == 2 and sc.anims[0][6] == 4 and sc.anims[1][6] == 1
    t = 0.5
    tg = sc.targets(t)
    left = sc.anims[0][0]
    np.testing.assert_allclose(tg[left], sc.x[left, :3] + [0, 0.5, 0], atol=1e-6)
    # materials: the cloth's own Lame parameters scaled by its thickness; the second part is one affine body
    mu, lam = S.lame(2e5, 0.3, 1e-3)
    np.testing.assert_allclose(sc.stretch_mu_lambda, [[mu, lam]] * len(sc.stretch_mu_lambda))
    assert np.all(sc.bending_stiffness == np.float32(0.1))
    assert sc.num_bodies == 1 and sc.num_verts == 50 + 4
    assert sc.offset[0] <= 0.5e-3 and sc.d_hat[0] <= 2e-3


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="REFERENCE_ROOT does not name the reference's sources")
def test_reference_scene_files_load():
    loaded = 0
    for f in sorted(glob.glob(REF + "/Scenes/*.json")):
        try:
            sc, st = scene_io.load_scene_json(f, [REF + "/InputMesh"])
        except FileNotFoundError:
            continue  # the 88K cylinder mesh is not in the reference's repository
        assert sc.num_verts > 0 and sc.faces.shape[0] > 0
        loaded += 1
        if os.path.basename(f) == "cloth_rotation_cylinder_7K.json":
            assert sc.pinned.sum() == 600 and len(sc.anims) == 2
            assert {round(a[3], 6) for a in sc.anims} == {round(math.radians(72), 6), round(-math.radians(72), 6)}
        if os.path.basename(f) == "cloth_rigid_coupling_drop.json":
            assert sc.num_bodies == 1 and sc.pinned.sum() == 4
    assert loaded >= 12


def _two_part_scene(tmp_path):
    _grid_obj(tmp_path / "grid.obj")
    scene = {"shells": [{"model_name": "grid.obj", "translation": [0, 1, 0]},
                        {"model_name": "grid.obj", "translation": [0.2, 1.1, 0.2], "scale": 0.1, "shell_type": "Rigid"}]}
    (tmp_path / "s.json").write_text(json.dumps(scene))
    return scene_io.load_scene_json(str(tmp_path / "s.json"), [str(tmp_path)])[0]


def test_state_file_round_trip_with_bodies(tmp_path):
    sc = _two_part_scene(tmp_path)
    rng = np.random.default_rng(3)
    x = sc.x.copy()
    x[:, :3] += rng.normal(0, 0.1, (sc.num_verts, 3)).astype(np.float32)
    v = np.zeros_like(x)
    v[:, :3] = rng.normal(0, 1, (sc.num_verts, 3)).astype(np.float32)
    p = tmp_path / "frame_3.state"
    scene_io.save_state(str(p), sc, x, v)
    text = p.read_text().splitlines()
    assert text[0] == "o position" and text.count("o q") == 1 and text.count("o qv") == 1
    assert len(text) == 4 + 2 * 50 + 2 * 4  # 50 mesh vertices, one body's four slots
    x2, v2 = scene_io.load_state(str(p), sc, like=sc.x)
    np.testing.assert_array_equal(x2[:, :3], x[:, :3])
    np.testing.assert_array_equal(v2[:, :3], v[:, :3])
    # the reference's 6-digit output reads too; a scene of another size is refused
    short = "\n".join(ln if not ln.startswith("v ") else "v " + " ".join(f"{float(t):g}" for t in ln.split()[1:])
                      for ln in text)
    (tmp_path / "short.state").write_text(short + "\n")
    x3, _ = scene_io.load_state(str(tmp_path / "short.state"), sc)
    np.testing.assert_allclose(x3[:, :3], x[:, :3], rtol=1e-5, atol=1e-6)
    (tmp_path / "bad.state").write_text("\n".join(text[:-1]) + "\n")
    with pytest.raises(ValueError):
        scene_io.load_state(str(tmp_path / "bad.state"), sc)
    with pytest.raises(FileNotFoundError):
        scene_io.load_state(str(tmp_path / "missing.state"), sc)


def test_frame_obj_round_trip(tmp_path):
    sc = _two_part_scene(tmp_path)
    p = tmp_path / "frame_0.obj"
    scene_io.write_obj(str(p), sc, sc.x)
    assert p.read_text().count("o mesh_") == 2
    x, f = scene_io.read_obj(str(p))
    np.testing.assert_array_equal(x, sc.x[:50, :3])
    np.testing.assert_array_equal(f, sc.faces[:, :3])
