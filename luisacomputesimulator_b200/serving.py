"""Serving form: drape requests admitted by free device memory and batched as they arrive.

A request is one scene advanced a fixed number of time steps (a "drape solve").  The server keeps
a queue of arrived requests; whenever a slot is free and the memory budget allows, it admits every
queued request that fits into a new ``NewtonBatch`` (state, trees and matrices stay resident on the
device for the whole solve) and steps it on its own CUDA stream from its own host thread, so
batches admitted at different times run on the GPU at the same time.  A batch's requests finish
together; their slot and memory are then given to the requests that arrived meanwhile.  Each
request's trajectory is the one it would have alone (the batched solver's per-scene independence).

The device-memory need of a batch is estimated from its vertex count with a per-vertex footprint
that the server measures on the batches it creates (cudaMemGetInfo before and after creation).
"""
from __future__ import annotations

import dataclasses
import threading
import time

import numpy as np
import torch

from .newton import NewtonBatch


@dataclasses.dataclass
class Request:
    rid: int
    scene: object
    arrival: float            # seconds after the start of the run
    steps: int = 20
    admitted: float = -1.0
    done: float = -1.0
    x: np.ndarray = None      # final positions (float32, V x 4)
    batch_size: int = 0
    rejected: bool = False    # larger than the whole memory budget

    @property
    def latency(self):
        return self.done - self.arrival


class Server:
    """Continuous batching of drape solves on one GPU.

    budget_bytes: device memory the server may hold (admission by free HBM against it);
    max_batches: batches stepping at the same time (one host thread and one stream each);
    max_batch_verts: vertices in one batch."""

    def __init__(self, budget_bytes=150e9, max_batches=2, max_batch_verts=1_500_000, cluster=0,
                 bytes_per_vertex=4096.0, device=0, solve=None, free_bytes=None, gather_s=0.4):
        self.budget = float(budget_bytes)
        self.max_batches = int(max_batches)
        self.max_batch_verts = int(max_batch_verts)
        self.cluster = cluster
        self.bpv = float(bytes_per_vertex)  # refined from measurements
        self.device = device
        # the batch runner and the free-memory query (replaceable, e.g. by fakes in host-only tests)
        # admission: requests that arrive within gather_s of the oldest queued one are batched with it
        self.gather_s = float(gather_s)
        self.solve = solve or self._solve_gpu
        self.free_bytes = free_bytes or (lambda: torch.cuda.mem_get_info()[0])
        self.lock = threading.Lock()
        self.reserved = 0.0
        self.active = 0
        self.peak_active = 0
        self.peak_reserved = 0.0
        self.launched = []
        self.log = []

    def _estimate(self, reqs):
        return self.bpv * sum(r.scene.num_verts for r in reqs)

    def _solve_gpu(self, reqs):
        """Creates the batch on its own stream, steps it, returns the final positions of every request."""
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            free0 = torch.cuda.mem_get_info()[0]
            batch = NewtonBatch([r.scene for r in reqs], cluster=self.cluster, stream=stream.cuda_stream)
            used = free0 - torch.cuda.mem_get_info()[0]
            with self.lock:  # refine the footprint estimate (concurrent creations make it approximate)
                v = sum(r.scene.num_verts for r in reqs)
                if used > 0:
                    self.bpv = max(self.bpv * 0.5 + 0.5 * used / v, 1024.0)
            for _ in range(reqs[0].steps):
                batch.step()
            xs = [batch.positions(k) for k in range(len(reqs))]
            del batch
        return xs

    def _run_batch(self, reqs, t0, est):
        try:
            start = time.perf_counter() - t0
            xs = self.solve(reqs)
            now = time.perf_counter() - t0
            with self.lock:
                self.log.append(dict(start=start, done=now, n=len(reqs), verts=sum(r.scene.num_verts for r in reqs)))
            for r, x in zip(reqs, xs):
                r.x, r.done, r.batch_size = x, now, len(reqs)
        finally:
            with self.lock:
                self.reserved -= est
                self.active -= 1

    def run(self, requests, poll_s=5e-4):
        """Serves `requests` (arrival times relative to the call) and returns them completed."""
        pending = sorted(requests, key=lambda r: r.arrival)
        queue, threads = [], []
        t0 = time.perf_counter()
        i = 0
        while i < len(pending) or queue or any(t.is_alive() for t in threads):
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i].arrival <= now:
                queue.append(pending[i])
                i += 1
            # a request larger than the whole budget can never be admitted
            while queue and self.bpv * queue[0].scene.num_verts > self.budget:
                queue[0].rejected = True
                queue.pop(0)
            if queue:
                with self.lock:
                    can = self.active < self.max_batches
                    free = self.free_bytes()
                    room = min(self.budget - self.reserved, free * 0.9)
                waited = now - queue[0].arrival
                more = i < len(pending) and pending[i].arrival - queue[0].arrival <= self.gather_s
                if can and (waited >= self.gather_s or not more):
                    cap = self.max_batch_verts
                    take, verts = [], 0
                    for r in queue:  # admit in arrival order while the memory budget allows
                        est = self.bpv * r.scene.num_verts
                        if take and (verts + r.scene.num_verts > cap or self._estimate(take) + est > room):
                            break
                        if not take and self._estimate(take) + est > room:
                            break
                        take.append(r)
                        verts += r.scene.num_verts
                    if not take and self.active == 0:
                        take = queue[:1]  # nothing running: the head fits the budget, so start it
                    if take:
                        est = self._estimate(take)
                        with self.lock:
                            self.reserved += est
                            self.active += 1
                            self.peak_active = max(self.peak_active, self.active)
                            self.peak_reserved = max(self.peak_reserved, self.reserved)
                        for r in take:
                            r.admitted = now
                        queue = queue[len(take):]
                        th = threading.Thread(target=self._run_batch, args=(take, t0, est), daemon=True)
                        th.start()
                        threads.append(th)
                        self.launched.append(len(take))
                        continue
            time.sleep(poll_s)
        for th in threads:
            th.join()
        return pending


def poisson_drapes(n, rate_hz, seed, v_min=2000, v_max=64000, steps=20):
    """n drape requests with Poisson arrivals at rate_hz: square cloth grids of log-uniform vertex count over
    a sphere or a box collider (seeded)."""
    from .scenes import random_cloth_scene
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n))
    t -= t[0]
    out = []
    for k in range(n):
        v = int(round(np.exp(rng.uniform(np.log(v_min), np.log(v_max)))))
        coll = "sphere" if rng.uniform() < 0.5 else "box"
        out.append(Request(k, random_cloth_scene(v, int(rng.integers(1 << 30)), coll), float(t[k]), steps))
    return out


def fifo_latencies(arrivals, service):
    """Latencies of a one-at-a-time first-in-first-out server with the given service times."""
    done, lat = 0.0, []
    for a, s in zip(arrivals, service):
        start = max(a, done)
        done = start + s
        lat.append(done - a)
    return np.array(lat)
