"""Host logic of the serving loop (no GPU): admission in arrival order against the memory budget,
bounded concurrency, continuous admission of late arrivals, rejection of requests larger than the budget,
and the one-at-a-time FIFO latency model."""
import threading
import time
import types

import numpy as np

from luisacomputesimulator_b200.serving import Request, Server, fifo_latencies


def _req(k, verts, arrival, steps=3):
    return Request(k, types.SimpleNamespace(num_verts=verts), arrival, steps)


class FakeGpu:
    """Stands in for the batched solver: sleeps in proportion to the batch size, records concurrency."""

    def __init__(self, per_vert_s=2e-7):
        self.per_vert_s = per_vert_s
        self.lock = threading.Lock()
        self.live = 0
        self.peak = 0
        self.batches = []

    def solve(self, reqs):
        with self.lock:
            self.live += 1
            self.peak = max(self.peak, self.live)
            self.batches.append([r.rid for r in reqs])
        time.sleep(0.01 + self.per_vert_s * sum(r.scene.num_verts for r in reqs))
        with self.lock:
            self.live -= 1
        return [np.full((r.scene.num_verts, 4), r.rid, np.float32) for r in reqs]


def test_all_requests_served_in_arrival_order_within_limits():
    gpu = FakeGpu()
    reqs = [_req(k, 1000 + 500 * (k % 5), 0.004 * k) for k in range(30)]
    srv = Server(budget_bytes=40_000 * 4096.0, max_batches=3, max_batch_verts=12_000, solve=gpu.solve,
                 free_bytes=lambda: 1 << 40)
    out = srv.run(reqs)
    assert all(r.done > 0 and not r.rejected for r in out)
    assert all(r.latency >= 0 and r.admitted >= r.arrival for r in out)
    assert gpu.peak <= 3 and srv.peak_active <= 3
    assert srv.peak_reserved <= srv.budget
    for b in gpu.batches:
        assert sum(1000 + 500 * (k % 5) for k in b) <= 12_000
    flat = [k for b in gpu.batches for k in b]
    assert flat == sorted(flat)  # admitted in arrival order
    assert sum(len(b) for b in gpu.batches) == 30 and len(gpu.batches) > 1
    assert all(np.all(r.x == r.rid) for r in out)  # every request gets its own result


def test_late_arrivals_join_while_others_run():
    gpu = FakeGpu(per_vert_s=2e-5)  # ~0.2 s per 10K-vertex batch
    reqs = [_req(0, 10_000, 0.0), _req(1, 1000, 0.05), _req(2, 1000, 0.06)]
    srv = Server(max_batches=2, gather_s=0.01, solve=gpu.solve, free_bytes=lambda: 1 << 40)
    out = srv.run(reqs)
    # request 0 runs alone; 1 and 2 arrive while it runs and are admitted before it finishes
    assert gpu.batches[0] == [0]
    assert out[1].admitted < out[0].done
    assert gpu.peak == 2


def test_memory_budget_limits_concurrency_and_rejects_oversize():
    gpu = FakeGpu(per_vert_s=1e-6)
    reqs = [_req(0, 1_000_000, 0.0), _req(1, 4000, 0.0), _req(2, 4000, 0.0), _req(3, 4000, 0.0)]
    srv = Server(budget_bytes=5000 * 4096.0, max_batches=4, solve=gpu.solve, free_bytes=lambda: 1 << 40)
    out = srv.run(reqs)
    assert out[0].rejected and out[0].done < 0
    assert all(r.done > 0 for r in out[1:])
    assert gpu.peak == 1  # one 4000-vertex request fits the budget at a time


def test_fifo_latency_model():
    lat = fifo_latencies([0.0, 0.1, 0.2, 5.0], [1.0, 1.0, 1.0, 1.0])
    np.testing.assert_allclose(lat, [1.0, 1.9, 2.8, 1.0])


def test_burst_within_gather_window_is_one_batch():
    gpu = FakeGpu(per_vert_s=1e-6)
    reqs = [_req(k, 2000, 0.001 * k) for k in range(8)]
    srv = Server(max_batches=4, gather_s=0.05, solve=gpu.solve, free_bytes=lambda: 1 << 40)
    srv.run(reqs)
    # the eight requests arrive within the gather window of the first one and run as one batch
    assert gpu.batches == [list(range(8))]
    assert len(srv.log) == 1 and srv.log[0]["n"] == 8
