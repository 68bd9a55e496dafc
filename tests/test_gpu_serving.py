"""Serving on the GPU: every request served through the continuous-batching loop equals the same request
solved alone bit for bit (the batches run with LCS_NEWTON_DETERMINISTIC: every sum in a fixed order) and stays
intersection-free."""
import numpy as np
import pytest

from luisacomputesimulator_b200 import scenes as S
from luisacomputesimulator_b200.newton import NewtonBatch
from luisacomputesimulator_b200.serving import Request, Server
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_served_requests_equal_alone():
    sizes = [(500, "sphere"), (900, "box"), (1200, "sphere"), (700, "box"), (400, "sphere")]
    reqs = [Request(k, S.random_cloth_scene(v, 40 + k, coll), 0.002 * k, steps=4) for k, (v, coll) in enumerate(sizes)]
    srv = Server(max_batches=2)
    out = srv.run(reqs)
    assert all(r.done > 0 and not r.rejected for r in out)
    assert sum(srv.launched) == len(reqs)
    for r in out:
        b = NewtonBatch([r.scene])
        for _ in range(r.steps):
            b.step()
        xa = b.positions(0)
        scale = np.abs(xa[:, :3] - r.scene.x[:, :3]).max()
        assert scale > 0
        np.testing.assert_array_equal(r.x, xa)
        assert O.min_distance(r.scene, r.x) > 0.0
