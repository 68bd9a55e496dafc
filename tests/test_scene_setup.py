"""Contact offset / d_hat set-up of the scenes (init_collision_data.cpp:67-171), on the CPU."""
import numpy as np

from luisacomputesimulator_b200 import scenes as S

f32 = np.float32


def test_scaling_rule_cases():
    # nothing to scale: offset + d_hat below 0.9 x the smallest rest distance
    assert S.scaled_offset_d_hat(0.0, 1e-3, 1.7e-3, rigid=False) == (0.0, float(f32(1e-3)))
    # d_hat cut to the safe distance (the 1 mm-spaced mesh: safe = 0.9 mm)
    so, sd = S.scaled_offset_d_hat(0.0, 1e-3, 1e-3, rigid=False)
    assert so == 0.0 and sd == float(f32(0.9) * f32(1e-3))
    # offset cut to half the safe distance first, then d_hat to what is left
    safe = f32(0.9) * f32(1.7e-3)
    so, sd = S.scaled_offset_d_hat(2e-3, 1e-3, 1.7e-3, rigid=False)
    assert so == float(f32(0.5) * safe) and sd == float(safe - f32(0.5) * safe)
    # a thin offset survives, d_hat takes the rest
    so, sd = S.scaled_offset_d_hat(4e-4, 1e-3, 1e-3, rigid=False)
    assert so == float(f32(2e-4)) and sd == float(f32(0.9) * f32(1e-3) - f32(2e-4))
    # a rigid body's safe distance is 1e8: never scaled
    assert S.scaled_offset_d_hat(2e-3, 1e-3, 1e-5, rigid=True) == (float(f32(1e-3)), float(f32(1e-3)))


def test_rigid_part_keeps_its_d_hat_while_a_soft_part_of_the_same_size_is_scaled():
    # a 1 mm box: its rest altitude (0.5 mm on the face diagonals' triangles) is far below d_hat
    bx, bf = S.box_mesh((1e-3, 1e-3, 1e-3), (0.0, 0.0, 0.0))
    cx, cf = S.cloth_grid(8, 8, 0.01, origin=(0.0, 0.05, 0.0), jitter=0.0)
    for rigid in (True, False):
        sc = S.assemble("box", [S.MeshPart(cx, cf, np.zeros(cx.shape[0], bool)),
                                S.MeshPart(bx, bf, np.zeros(8, bool), rigid=rigid, thickness=2e-4)],
                        dt=1 / 60, gravity=(0, -9.8, 0), kappa=1e7)
        box = slice(cx.shape[0], cx.shape[0] + 8)
        cloth = slice(0, cx.shape[0])
        assert (sc.d_hat[cloth] == f32(1e-3)).all() and (sc.offset[cloth] == 0.0).all()
        if rigid:
            assert (sc.d_hat[box] == f32(1e-3)).all() and (sc.offset[box] == f32(1e-4)).all()
        else:
            assert (sc.d_hat[box] < f32(1e-3)).all()
            assert (sc.offset[box] + sc.d_hat[box] < f32(1e-3)).all()
