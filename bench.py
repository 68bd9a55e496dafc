#!/usr/bin/env python
"""Newton iterations/s on the 88,800-vertex twisted cloth tube.

Workload: a 300 x 296 periodic tube (88,800 vertices, 177,000 faces, 265,800 edges), radius
0.15 m, length 0.6 m, the two end rings pinned and rotated at -/+2 rad/s about the tube axis;
dt = 1/100 s, d_hat = 1e-3 m, thickness 0, kappa = 1e9, 3 Newton iterations per step,
Jacobi-PCG up to 100 iterations / relative residual 1e-4, CCD line search.  Synthetic, seeded
geometry (no mesh file).  A bench step is one time step; the metric counts the Newton
iterations those steps ran.  State stays on the GPU; the working set (~150 MB: BVHs,
candidate lists, block matrix) is larger than L2 and L2 is also flushed between steps.

--impl reference runs the CPU restatement of the same Newton iteration (the oracle, OpenMP on
all host cores) on the tube at the state the 60-step run reaches (end rings at -/+1.2 rad).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton iters/s at 88K-vert cloth"
UNIT = "newton_iters/s"
L2_BYTES = 126 * 1024 * 1024


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=57)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--mode", choices=["fused", "plain"], default="fused")
    p.add_argument("--fp64", action="store_true", help="precision form")
    p.add_argument("--pcg", choices=["rows", "cg1", "cg1-global"], default="cg1",
                   help="fused mode: row-resident PCG (classic recurrences: 3 grid syncs/iter; cg1: the "
                        "single-reduction form, slice-resident where the rows fit -- one block per SM with its "
                        "leading matrix groups in shared memory; cg1-global: the single-reduction form reading "
                        "the matrix from L2 every iteration)")
    p.add_argument("--traversal", choices=["fast", "full"], default="fast",
                   help="fast: DCD lists filtered from the previous iteration's CCD lists (same sets); "
                        "full: a traversal for every list")
    p.add_argument("--e2e-steps", type=int, default=10)
    p.add_argument("--cpu-iters", type=int, default=0, help="CPU baseline sample (0: auto, ~10-30 s)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--n-around", type=int, default=300)
    p.add_argument("--n-along", type=int, default=296)
    p.add_argument("--workload", choices=["tube", "batch", "serve"], default="tube",
                   help="tube: the headline Newton iters/s line; batch: batched drape solves/s (256 scenes); "
                        "serve: Poisson drape requests, p50/p99 latency and solves/s")
    p.add_argument("--n-scenes", type=int, default=256, help="batch workload: cloth-on-sphere scenes")
    p.add_argument("--n-box-scenes", type=int, default=16,
                   help="batch workload: cloth scenes coupled with an affine rigid box (12 DOFs, 8 vertices)")
    p.add_argument("--solve-steps", type=int, default=20, help="time steps of one drape solve")
    p.add_argument("--plain-sample", type=int, default=32, help="requests/scenes timed through the plain loop")
    p.add_argument("--requests", type=int, default=64, help="serve workload: requests")
    p.add_argument("--rate", type=float, default=200.0, help="serve workload: Poisson arrival rate (1/s)")
    p.add_argument("--max-batches", type=int, default=2, help="serve workload: batches in flight")
    p.add_argument("--gather", type=float, default=0.4, help="serve workload: admission gather window (s)")
    p.add_argument("--no-plain", action="store_true", help="batch/serve: skip the plain-loop comparator")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def tube_config(a):
    return {"workload": f"twisted tube {a.n_around}x{a.n_along} ({a.n_around * a.n_along} verts), 60-step run, "
                        "rings -/+2 rad/s, dt 1/100, d_hat 1e-3, kappa 1e9, 3 Newton/step, PCG <=100 it rel 1e-4",
            "verts": a.n_around * a.n_along, "dt": 0.01, "d_hat": 1e-3, "kappa": 1e9, "newton_per_step": 3,
            "pcg": "Jacobi, max 100 iterations, rel 1e-4", "l2": "flushed between steps (256 MB write)"}


# --------------------------------------------------------------------------- clocks sampling
class Clocks:
    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.index = index

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                                       "200", "-i", str(self.index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for ln in open(self.f.name):
                parts = [s.strip() for s in ln.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(kernel):
    """DRAM bytes per launch of the tube's PCG kernel from the committed ncu capture (or None)."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_tube88k_traffic.txt")
    try:
        for ln in open(path):
            if ln.startswith("bytes_per_launch="):
                return float(ln.split("=")[1])
    except Exception:
        return None
    return None


# ------------------------------------------------------------------------------ CPU baseline
def cpu_sample(a, iters=0, budget_s=20.0):
    """Newton iterations/s of the oracle (CPU restatement) on the tube state of the 60-step run."""
    import numpy as np

    from oracle import newton_cpu as N
    from tests import scenarios as SC
    sc, x = SC.twisted_tube_state(angle=1.2, n_around=a.n_around, n_along=a.n_along)
    pat = N.MaterialPattern(sc)
    xt = x.copy()
    done, t0 = 0, time.perf_counter()
    while True:
        x, toi, st, cnt = N.newton_iteration(sc, x, xt, sc.dt, pattern=pat)
        done += 1
        el = time.perf_counter() - t0
        if (iters and done >= iters) or (not iters and (el > budget_s or done >= 20)):
            break
    cores = os.cpu_count()
    return done / el, done, el, cores, np.float32(toi)


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import numpy as np

    from oracle import newton_cpu as N
    from tests import scenarios as SC
    sc, x = SC.twisted_tube_state(angle=1.2, n_around=a.n_around, n_along=a.n_along)
    pat = N.MaterialPattern(sc)
    xt = x.copy()
    for _ in range(a.warmup):
        N.newton_iteration(sc, x, xt, sc.dt, pattern=pat)
    # one bench step = one Newton iteration of the CPU restatement (a bounded sample of the
    # 3-iteration time step); cap the timed count so the run ends within a few minutes
    steps = min(a.steps, 40)
    t0 = time.perf_counter()
    for _ in range(steps):
        x, toi, st, cnt = N.newton_iteration(sc, x, xt, sc.dt, pattern=pat)
    el = time.perf_counter() - t0
    v = steps / el
    cores = os.cpu_count()
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference", "config": tube_config(a),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{steps} Newton iterations of the CPU restatement (oracle, OpenMP) on the "
                                       "tube at its 60-step state; one bench step = one Newton iteration"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    _ = np


# --------------------------------------------------------------------------------- our arm
def run_ours(a):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from luisacomputesimulator_b200 import _capi, scenes
    from luisacomputesimulator_b200.newton import NewtonSolver

    lib = _capi.load()
    _capi.check(lib.lcs_device_check(local), "device check")
    sc = scenes.twisted_tube(a.n_around, a.n_along)
    solver = NewtonSolver(sc, plain=(a.mode == "plain"), fp64=a.fp64, profile=True, single_reduction=(a.pcg != "rows"),
                          global_matrix=(a.pcg == "cg1-global"), full_traversal=(a.traversal == "full"))
    stream = torch.cuda.current_stream()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    for _ in range(a.warmup):
        solver.step()
    torch.cuda.synchronize()
    solver.reset_profile()
    if world > 1:
        torch.distributed.barrier()

    newton, pcg, ms_total = 0, 0, 0.0
    per_step = []
    launches0 = lib.lcs_launch_count()
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = solver.step()
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            per_step.append((ms, st.newton_iters, st.retries, st.host_ms))
            ms_total += ms
            newton += st.newton_iters
            pcg += st.pcg_iters
    launches = lib.lcs_launch_count() - launches0
    torch.cuda.synchronize()
    clocks = clk.summary()
    prof = solver.profile()
    last = dict(vf=st.vf_candidates, ee=st.ee_candidates, pairs=st.contact_pairs, ccd_vf=st.ccd_vf_candidates,
                ccd_ee=st.ccd_ee_candidates, last_toi=st.last_toi, last_rel_residual=st.last_rel_residual)
    cnt = solver.counts()

    # end to end through the public host-buffer call (x, v in from pinned host, x, v out)
    V = sc.num_verts
    hx = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    hv = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    hx.numpy()[:] = solver.positions()
    hv.numpy()[:] = solver.velocities()
    e2e_ms, e2e_newton = 0.0, 0
    for _ in range(a.e2e_steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s2 = solver.step_host(hx.numpy(), hv.numpy(), hx.numpy(), hv.numpy())
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        e2e_newton += s2.newton_iters

    # max over ranks of the time, sum of the work
    t_s = ms_total / 1e3
    e2e_s = e2e_ms / 1e3
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([t_s, e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        nn = torch.tensor([newton, e2e_newton], device="cuda", dtype=torch.float64)
        dist.all_reduce(nn, op=dist.ReduceOp.SUM)
        t_s, e2e_s = float(tt[0]), float(tt[1])
        newton_all, e2e_all = float(nn[0]), float(nn[1])
    else:
        newton_all, e2e_all = float(newton), float(e2e_newton)

    if rank == 0:
        value = newton_all / t_s
        solver_uses_rows = solver.uses_row_pcg()
        pcg_kernel_name = {"cg1-res": "k_pcg_res (single-reduction slice-resident Jacobi-PCG)",
                           "cg1": "k_pcg_cg1 (single-reduction row-resident Jacobi-PCG)",
                           "rows": "k_pcg_rows (row-resident Jacobi-PCG)"}[solver.pcg_kind()] if solver_uses_rows else \
            ("k_pcg_fused (persistent Jacobi-PCG solve)" if a.mode == "fused" else "plain PCG kernels")
        # roofline of the dominant kernel: the persistent PCG solve (one launch per Newton iteration)
        pcg_ms, pcg_launches = prof["pcg"]
        nnz = cnt["nnz_material"] + 12 * last["pairs"]
        it_per_launch = pcg / max(pcg_launches, 1)
        # algorithmic bytes of one PCG iteration: every matrix block once (36 B values + 4 B
        # column), the diagonal blocks (48 B/row) and the exchanged direction written and read
        # once (32 B/row) when the row state stays in registers (row-resident kernels); the
        # CSR-vector kernel also streams r, z, p, q, x (312 B/row in all)
        rows_kind = a.mode == "fused" and solver_uses_rows
        bytes_per_iter = 40.0 * nnz + (80.0 if rows_kind else 312.0) * V
        bytes_per_launch = it_per_launch * bytes_per_iter + 160.0 * V
        achieved = bytes_per_launch / (pcg_ms / max(pcg_launches, 1) / 1e3) / 1e9
        peak, peak_kind = measured_peak()
        traffic = committed_traffic(pcg_kernel_name.split()[0])
        cpu = None
        if not a.no_cpu_baseline and world == 1:
            v_cpu, n_cpu, el_cpu, cores, _ = cpu_sample(a, a.cpu_iters)
            cpu = {"value": v_cpu, "unit": UNIT, "cores": cores, "kind": "port",
                   "sample": f"{n_cpu} Newton iterations ({el_cpu:.1f} s) of the CPU restatement (oracle, OpenMP, "
                             "all host cores) on the tube at its 60-step state"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_total / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" + ("+f64 reductions" if a.fp64 else ""), "data": "synthetic (seeded tube mesh)",
            "impl": "ours", "mode": a.mode, "pcg": solver.pcg_kind(), "traversal": a.traversal,
            "config": {**tube_config(a), "parallelism": f"replicas x{world}" if world > 1 else "single scene"},
            "e2e": None if a.e2e_steps == 0 else {
                "value": e2e_all / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 16 * V,
                "d2h_bytes_per_step": 2 * 16 * V, "steps": a.e2e_steps},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": pcg_kernel_name,
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "pcg_iters_per_launch": it_per_launch, "avg_launch_ms": pcg_ms / max(pcg_launches, 1)},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "newton_iters": newton, "pcg_iters": pcg,
            "step_ms": {"min": min(p[0] for p in per_step), "median": statistics.median(p[0] for p in per_step),
                        "max": max(p[0] for p in per_step), "retries": sum(p[2] for p in per_step),
                        "host_ms_median": statistics.median(p[3] for p in per_step)},
            "phase_ms": {k: round(v[0], 3) for k, v in prof.items()},
            "last_step": last,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    _ = np


# ------------------------------------------------------------------------- batching / serving
def _log_uniform_sizes(n, lo, hi, seed):
    import numpy as np
    rng = np.random.default_rng(seed)
    return [int(round(v)) for v in np.exp(rng.uniform(np.log(lo), np.log(hi), n))]


def _plain_service(scene, steps, plain=True):
    """Wall time of one drape solve through the one-scene-at-a-time loop (create, steps, read back)."""
    import torch
    from luisacomputesimulator_b200.newton import NewtonSolver
    torch.cuda.synchronize()
    t = time.perf_counter()
    s = NewtonSolver(scene, plain=plain)
    for _ in range(steps):
        s.step()
    s.positions()
    del s
    return time.perf_counter() - t


def _stratified(items, key, k):
    order = sorted(range(len(items)), key=lambda i: key(items[i]))
    if k >= len(items):
        return order
    return [order[int((j + 0.5) * len(items) / k)] for j in range(k)]


def run_batch(a):
    """Batching form: n_scenes cloth-on-sphere drapes (vertex counts log-uniform in [1K, 32K], seeds 0..n-1)
    stepped together for solve_steps time steps; against the plain one-scene-at-a-time loop."""
    import numpy as np
    import torch
    from luisacomputesimulator_b200 import _capi, scenes
    from luisacomputesimulator_b200.newton import NewtonBatch
    from luisacomputesimulator_b200.sharding import combine, partition
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lib = _capi.load()
    _capi.check(lib.lcs_device_check(local), "device check")
    sizes = list(_log_uniform_sizes(a.n_scenes, 1000, 32000, seed=0))
    sizes += list(_log_uniform_sizes(a.n_box_scenes, 1000, 32000, seed=1)) if a.n_box_scenes else []
    n_all = len(sizes)
    V_all = int(sum(sizes))
    # whole scenes per rank (independent problems: no collective on the data path)
    mine = partition(sizes, world)[rank]
    scs = [scenes.random_cloth_scene(sizes[k], k, "sphere") if k < a.n_scenes else
           scenes.cloth_box_scene(sizes[k], k) for k in mine]
    V = sum(sc.num_verts for sc in scs)
    warm = NewtonBatch(scs[:4])  # warm-up: first-call set-up paths
    for _ in range(max(a.warmup, 1)):
        warm.step()
    del warm
    torch.cuda.synchronize()
    t_e2e = time.perf_counter()
    batch = NewtonBatch(scs)
    t_create = time.perf_counter() - t_e2e
    launches0 = lib.lcs_launch_count()
    newton = 0
    stream = torch.cuda.current_stream()
    with Clocks(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t_steps = time.perf_counter()
        for _ in range(a.solve_steps):
            st = batch.step()
            newton += st.newton_iters
        e1.record(stream)
        e1.synchronize()
        t_steps = time.perf_counter() - t_steps
    launches = lib.lcs_launch_count() - launches0
    clocks = clk.summary()
    xs = [batch.positions(k) for k in range(len(scs))]
    t_e2e = time.perf_counter() - t_e2e
    assert all(np.isfinite(x).all() for x in xs)
    tuned_chunks, tuned_ms = batch.pcg_tuning()
    del batch
    ms = e0.elapsed_time(e1)
    done_all, t_max = combine(len(scs), ms / 1e3, device="cuda")  # sum of solves, max of device time
    _, e2e_max = combine(len(scs), t_e2e, device="cuda")
    _, launches_max = combine(0, float(launches), device="cuda")
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    no_plain = a.no_plain
    sample = [] if no_plain else _stratified(scs, lambda sc: sc.num_verts, a.plain_sample)
    plain_t = [_plain_service(scs[i], a.solve_steps, plain=True) for i in sample] or [float("nan")]
    fused_t = [_plain_service(scs[i], a.solve_steps, plain=False) for i in sample] or [float("nan")]
    value = done_all / t_max
    line = {
        "metric": f"batched drape solves/s ({a.n_scenes} cloth-on-sphere + {a.n_box_scenes} cloth-box scenes, 1K-32K "
                  f"verts, {a.solve_steps} steps)",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.solve_steps, "warmup": max(a.warmup, 1),
        "ms_per_step": 1e3 * t_max / a.solve_steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded cloth grids over icospheres)", "impl": "ours",
        "config": {"workload": f"C4 batching: {a.n_scenes} cloth-on-sphere scenes (cloth sizes log-uniform [1K, 32K], "
                               f"seed 0) + {a.n_box_scenes} scenes of a cloth (sizes seed 1) over a sphere with an "
                               f"affine rigid box (8 verts, 12 DOFs) dropped on it; {V_all} cloth vertices in all, "
                               "scene k seeded k, dt 1/60, kappa 1e7, 3 Newton/step, PCG <=100 it rel 1e-4",
                   "scenes": n_all, "verts_rank0": V, "pcg_cluster": "auto",
                   "pcg_autotune": {"chunks_per_cta": tuned_chunks, "tuned_solve_ms": tuned_ms,
                                    "candidates": [2, 4, 8, 16]},
                   "parallelism": f"whole scenes over {world} GPUs" if world > 1 else "one batch"},
        "e2e": {"value": done_all / e2e_max, "unit": "solves/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": 16 * V, "includes": "batch creation (host upload), all steps, read-back"},
        "gpu_launches": int(launches_max), "newton_iters": newton, "create_s": t_create,
        "plain_loop": {"value": 1.0 / float(np.mean(plain_t)), "unit": "solves/s", "sample": len(sample),
                       "kind": "plain one-scene-at-a-time GPU loop (reference dispatch structure), create + steps + "
                               "read-back per scene, size-stratified sample"},
        "fused_single_loop": {"value": 1.0 / float(np.mean(fused_t)), "unit": "solves/s", "sample": len(sample)},
        "clocks": clocks,
    }
    if no_plain:
        line["plain_loop"] = line["fused_single_loop"] = None
        line["ratio_vs_plain"] = None
    else:
        line["ratio_vs_plain"] = line["value"] / line["plain_loop"]["value"]
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_serve(a):
    """Serving form: Poisson drape requests (2K-64K verts, sphere or box collider, solve_steps steps) through
    the continuous-batching server; p50/p99 latency and solves/s against the one-at-a-time plain loop."""
    import numpy as np
    import torch
    from luisacomputesimulator_b200 import _capi
    from luisacomputesimulator_b200.newton import NewtonBatch
    from luisacomputesimulator_b200.serving import Server, fifo_latencies, poisson_drapes
    torch.cuda.set_device(0)
    lib = _capi.load()
    _capi.check(lib.lcs_device_check(0), "device check")
    warm = poisson_drapes(3, a.rate, seed=99, v_max=4000, steps=2)
    Server(max_batches=2).run(warm)
    reqs = poisson_drapes(a.requests, a.rate, seed=0, steps=a.solve_steps)
    server = Server(max_batches=a.max_batches, gather_s=a.gather)
    launches0 = lib.lcs_launch_count()
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        done = [r for r in server.run(reqs) if not r.rejected and r.done >= 0]
        wall = time.perf_counter() - t0
    launches = lib.lcs_launch_count() - launches0
    clocks = clk.summary()
    lat = np.array([r.latency for r in done])
    span = max(r.done for r in done) - min(r.arrival for r in done)
    # alone == in the mix: two requests re-run alone through the same batched solver, and one of them alone
    # twice (the run-to-run spread that float atomics alone produce over the solve)
    dev, rerun = [], []
    for r in done[:2]:
        xs = []
        for _ in range(2):
            b = NewtonBatch([r.scene])
            for _ in range(r.steps):
                b.step()
            xs.append(b.positions(0))
            del b
        scale = max(float(np.abs(xs[0][:, :3] - r.scene.x[:, :3]).max()), 1e-12)
        dev.append(float(np.abs(xs[0][:, :3] - r.x[:, :3]).max() / scale))
        rerun.append(float(np.abs(xs[0][:, :3] - xs[1][:, :3]).max() / scale))
    sample = _stratified(done, lambda r: r.scene.num_verts, 1 if a.no_plain else min(a.plain_sample, len(done)))
    service = {i: _plain_service(done[i].scene, a.solve_steps, plain=True) for i in sample}
    mean_service = float(np.mean(list(service.values())))
    # one-at-a-time FIFO over the same arrivals; requests outside the timed sample get the sample mean
    plain_lat = fifo_latencies([r.arrival for r in done], [service.get(i, mean_service) for i in range(len(done))])
    line = {
        "metric": f"served drape solves/s ({len(done)} Poisson requests at {a.rate:g}/s, 2K-64K verts)",
        "value": len(done) / span, "unit": "solves/s", "n_gpus": 1, "steps": a.solve_steps, "warmup": 1,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded cloth grids over icospheres / boxes)", "impl": "ours",
        "config": {"workload": f"C5 serving: {len(done)} requests, Poisson {a.rate:g}/s (seed 0), cloth 2K-64K verts "
                               f"log-uniform over a sphere or box, {a.solve_steps} steps each, admission by free HBM "
                               f"against a 150 GB budget, up to {a.max_batches} batches in flight, gather window "
                               f"{a.gather:g} s", "requests": len(done)},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "batches": [{k: round(v, 3) if isinstance(v, float) else v for k, v in b.items()} for b in server.log],
        "wall_s": wall, "gpu_launches": int(launches),
        "alone_vs_mix_max_rel_dev": max(dev) if dev else None,
        "alone_vs_alone_max_rel_dev": max(rerun) if rerun else None,
        "plain_loop": {"value": 1.0 / mean_service, "unit": "solves/s",
                       "latency_s": {"p50": float(np.percentile(plain_lat, 50)),
                                     "p99": float(np.percentile(plain_lat, 99))},
                       "sample": len(sample),
                       "kind": "plain one-at-a-time GPU loop; service times measured on a size-stratified sample, "
                               "FIFO queue over the same arrivals"},
        "e2e": {"value": len(done) / span, "unit": "solves/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "includes": "request admission, host upload, all steps, read-back of every request"},
        "clocks": clocks,
    }
    line["ratio_vs_plain"] = line["value"] / line["plain_loop"]["value"]
    print(json.dumps(line), flush=True)


def main():
    a = args_()
    if a.workload == "batch" and a.impl == "ours":
        return run_batch(a)
    if a.workload == "serve" and a.impl == "ours":
        return run_serve(a)
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
