#!/usr/bin/env python
"""Newton iterations/s on the 88,800-vertex twisted cloth tube.

Workload: a 300 x 296 periodic tube (88,800 vertices, 177,000 faces, 265,800 edges), radius 0.15 m,
length 0.6 m, the two end rings pinned and rotated at -/+2 rad/s about the tube axis; dt = 1/100 s,
d_hat = 1e-3 m, thickness 0, kappa = 1e9, 3 Newton iterations per step, Jacobi-PCG with at most
100 iterations (stop at r.z < 1e-10 or |r| <= 1e-4 |r0|), CCD line search.  Synthetic, seeded geometry
(no mesh file).  Every bench step is the same time step: the one after the state the run from rest
reaches after FRAME steps (tests/golden/tube88k_state.npz, made on the CPU by the restatement of the
Newton loop), loaded before the step outside the timed region.  The metric counts the Newton
iterations those steps ran.  The working set (~150 MB: BVHs, candidate lists, block matrix) is larger
than L2 and L2 is also flushed between steps.

--impl reference runs the CPU restatement of the same time step (the oracle, OpenMP on all host cores)
from the same state, with the same PCG stop rule.  --workload c1 is the small configuration: a 64 x 64
cloth dropped onto a pinned 2,562-vertex icosphere, 10 steps from rest, timed as whole 10-step runs.
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
METRIC_C1 = "Newton iters/s, 64x64 cloth on a pinned icosphere (C1)"
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
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-converged", action="store_true",
                   help="tube: skip the second measurement with the PCG run to |r| <= 1e-4 |r0|")
    p.add_argument("--converged-cap", type=int, default=2000,
                   help="tube: PCG iteration cap of the converged measurement")
    p.add_argument("--workload", choices=["tube", "c1", "batch", "serve"], default="tube",
                   help="tube: the headline Newton iters/s line; c1: the small cloth-on-icosphere configuration; "
                        "batch: batched drape solves/s (256 scenes); serve: Poisson drape requests, p50/p99 latency "
                        "and solves/s")
    p.add_argument("--n-scenes", type=int, default=256, help="batch workload: cloth-on-sphere scenes")
    p.add_argument("--n-box-scenes", type=int, default=16,
                   help="batch workload: cloth scenes coupled with an affine rigid box (12 DOFs, 8 vertices)")
    p.add_argument("--solve-steps", type=int, default=20, help="time steps of one drape solve")
    p.add_argument("--plain-sample", type=int, default=32, help="requests/scenes timed through the plain loop")
    p.add_argument("--requests", type=int, default=64, help="serve workload: requests")
    p.add_argument("--rate", type=float, default=200.0, help="serve workload: Poisson arrival rate (1/s)")
    p.add_argument("--max-batches", type=int, default=3, help="serve workload: batches in flight")
    p.add_argument("--gather", type=float, default=0.05,
                   help="serve workload: admission gather window (s); requests arriving while the batches in flight "
                        "run wait for a free slot and are admitted together")
    p.add_argument("--no-plain", action="store_true", help="batch/serve: skip the plain-loop comparator")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


PCG_RULE = "Jacobi-PCG, stop at r.z < 1e-10 or |r| <= 1e-4 |r0| (checked every iteration), at most {cap} iterations"


def tube_config(frame, cap=100):
    """The tube workload's config; both arms print the same dict."""
    return {"workload": f"twisted tube 300x296 (88800 verts): the time step after step {frame} of the run from rest "
                        "(rings -/+2 rad/s), the same state in every timed step and in both arms; dt 1/100, d_hat 1e-3, "
                        f"kappa 1e9, 3 Newton/step, {PCG_RULE.format(cap=cap)}",
            "verts": 88800, "frame": frame, "dt": 0.01, "d_hat": 1e-3, "kappa": 1e9, "newton_per_step": 3,
            "pcg": PCG_RULE.format(cap=cap), "state": "tests/golden/tube88k_state.npz (CPU restatement run from rest)",
            "l2": "flushed between steps (256 MB write)"}


def c1_config():
    return {"workload": "C1: 64x64 cloth (1 cm spacing, jitter seed 0) dropped from 5 cm onto a pinned 2562-vertex "
                        "icosphere (r 0.2 m), 10 steps from rest per bench step; dt 1/60, d_hat 1e-3, kappa 1e7, "
                        f"3 Newton/step, {PCG_RULE.format(cap=100)}",
            "verts": 6658, "dt": 1.0 / 60.0, "d_hat": 1e-3, "kappa": 1e7, "newton_per_step": 3, "sim_steps": 10,
            "pcg": PCG_RULE.format(cap=100), "l2": "working set (< 10 MB) fits L2; flushed between bench steps"}


def _residual_summary(recs):
    import numpy as np
    rel = np.array([r["rel_residual"] for r in recs], np.float64)
    it = np.array([r["pcg_iters"] for r in recs], np.float64)
    if not len(rel):
        return None
    return {"solves": int(len(rel)), "rel_residual_p50": float(np.median(rel)), "rel_residual_max": float(rel.max()),
            "pcg_iters_p50": float(np.median(it)), "pcg_iters_max": int(it.max()),
            "converged_1e-4": int((rel <= 1e-4).sum())}


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


# ------------------------------------------------------------------------------ CPU arm
def cpu_tube_steps(budget_s=20.0, max_steps=0, warmup=1, cap=100):
    """Newton iterations/s of the CPU restatement (oracle, OpenMP on all host cores) over whole time steps from
    the tube state, every step from the same state; returns (value, summary)."""
    from oracle import newton_cpu as N
    from tests import scenarios as SC
    sc, x, v, frame = SC.tube_state()
    pat = N.MaterialPattern(sc)
    run = lambda: N.time_step(sc, x, v, frame, pattern=pat, pcg_max_iter=cap, pcg_check_every=1)  # noqa: E731
    for _ in range(warmup):
        run()
    recs, el, steps = [], 0.0, 0
    while True:
        t0 = time.perf_counter()
        _, _, r = run()
        el += time.perf_counter() - t0
        recs += r
        steps += 1
        if (max_steps and steps >= max_steps) or (not max_steps and el > budget_s):
            break
    first = recs[0]
    return len(recs) / el, {"steps": steps, "newton_iters": len(recs), "seconds": el, "frame": frame,
                            "first_iteration": {k: first[k] for k in ("vf", "ee", "pairs")},
                            "residuals": _residual_summary(recs)}


def cpu_c1_runs(budget_s=15.0, max_runs=0, warmup=1):
    """Newton iterations/s of the CPU restatement over whole 10-step C1 runs from rest."""
    import numpy as np

    from luisacomputesimulator_b200 import scenes
    from oracle import newton_cpu as N
    sc = scenes.cloth_on_sphere(n=64)
    pat = N.MaterialPattern(sc)

    def run():
        x, v, out = sc.x.copy(), np.zeros_like(sc.x), []
        for f in range(10):
            x, v, r = N.time_step(sc, x, v, f, pattern=pat, pcg_check_every=1)
            out += r
        return out
    for _ in range(warmup):
        run()
    recs, el, runs = [], 0.0, 0
    while True:
        t0 = time.perf_counter()
        recs += run()
        el += time.perf_counter() - t0
        runs += 1
        if (max_runs and runs >= max_runs) or (not max_runs and el > budget_s):
            break
    return len(recs) / el, {"runs": runs, "newton_iters": len(recs), "seconds": el,
                            "residuals": _residual_summary(recs)}


def run_reference(a):
    """The reference arm: the CPU restatement of the reference's kernels on all host cores, the same workload,
    metric and config as the GPU arm; each bench step is a bounded sample (whole time steps)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count()
    if a.workload == "c1":
        v, info = cpu_c1_runs(budget_s=30.0, max_runs=min(a.steps, 20), warmup=min(a.warmup, 1))
        cfg, metric = c1_config(), METRIC_C1
        sample = f"{info['runs']} whole 10-step C1 runs ({info['newton_iters']} Newton iterations, {info['seconds']:.1f} s)"
    else:
        v, info = cpu_tube_steps(budget_s=30.0, max_steps=min(a.steps, 12), warmup=min(a.warmup, 1))
        cfg, metric = tube_config(info["frame"]), METRIC
        sample = (f"{info['steps']} time steps from the tube state ({info['newton_iters']} Newton iterations, "
                  f"{info['seconds']:.1f} s)")
    line = {"metric": metric, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": info.get("steps", info.get("runs")),
            "warmup": min(a.warmup, 1), "ms_per_step": 1e3 * info["seconds"] / max(info.get("steps", info.get("runs")), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample + " of the CPU restatement of the reference's kernels (oracle, OpenMP, "
                                                "all host cores); the reference's LuisaCompute build is unavailable"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "residuals": info["residuals"]}
    if "first_iteration" in info:
        line["first_iteration"] = info["first_iteration"]
    if a.workload != "c1" and not a.no_converged:
        vc, ic = cpu_tube_steps(budget_s=20.0, max_steps=2, warmup=0, cap=a.converged_cap)
        line["converged_1e-4"] = {"value": vc, "unit": UNIT, "pcg": PCG_RULE.format(cap=a.converged_cap),
                                  "steps": ic["steps"], "residuals": ic["residuals"]}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------- our arm
def _timed_tube_steps(solver, x4, v4, frame, steps, flush, stream, records=None):
    """`steps` time steps, each from (x4, v4) at `frame` (loaded outside the timed region, L2 flushed), each timed
    with CUDA events on the solver's stream; returns (device ms, Newton iterations, PCG iterations, per-step)."""
    import torch
    ms_total, newton, pcg, per = 0.0, 0, 0, []
    for _ in range(steps):
        solver.upload(x4, v4)
        solver.set_frame(frame)
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = solver.step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        per.append((ms, st.newton_iters, st.retries, st.host_ms))
        ms_total += ms
        newton += st.newton_iters
        pcg += st.pcg_iters
        if records is not None:
            records += solver.iteration_log()
    return ms_total, newton, pcg, per


def run_ours(a):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from luisacomputesimulator_b200 import _capi
    from luisacomputesimulator_b200.newton import NewtonSolver
    from tests import scenarios as SC

    lib = _capi.load()
    _capi.check(lib.lcs_device_check(local), "device check")
    sc, x4, v4, frame = SC.tube_state()
    mk = lambda cap: NewtonSolver(sc, plain=(a.mode == "plain"), fp64=a.fp64, profile=True,  # noqa: E731
                                  single_reduction=(a.pcg != "rows"), global_matrix=(a.pcg == "cg1-global"),
                                  full_traversal=(a.traversal == "full"), pcg_max_iter=cap)
    solver = mk(100)
    stream = torch.cuda.current_stream()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    _timed_tube_steps(solver, x4, v4, frame, a.warmup, flush, stream)
    torch.cuda.synchronize()
    solver.reset_profile()
    if world > 1:
        torch.distributed.barrier()

    recs = []
    launches0 = lib.lcs_launch_count()
    with Clocks(local) as clk:
        ms_total, newton, pcg, per_step = _timed_tube_steps(solver, x4, v4, frame, a.steps, flush, stream, recs)
    launches = lib.lcs_launch_count() - launches0
    torch.cuda.synchronize()
    clocks = clk.summary()
    prof = solver.profile()
    cnt = solver.counts()
    first = recs[0]

    # end to end through the public host-buffer call: x, v in from pinned host memory, x, v out; every step
    # from the same state (wall clock around the call, which synchronises)
    V = sc.num_verts
    hx_in = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    hv_in = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    hx_out = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    hv_out = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    hx_in.numpy()[:] = x4
    hv_in.numpy()[:] = v4
    e2e_s, e2e_newton = 0.0, 0
    for k in range(a.e2e_steps + 1):
        solver.set_frame(frame)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2 = solver.step_host(hx_in.numpy(), hv_in.numpy(), hx_out.numpy(), hv_out.numpy())
        el = time.perf_counter() - t0
        if k:  # the first call is a warm-up
            e2e_s += el
            e2e_newton += s2.newton_iters

    conv = None
    if not a.no_converged:  # the same steps with the PCG run to |r| <= 1e-4 |r0| (cap raised)
        del solver
        solver = mk(a.converged_cap)
        _timed_tube_steps(solver, x4, v4, frame, 2, flush, stream)
        crecs = []
        cms, cnewton, cpcg, _ = _timed_tube_steps(solver, x4, v4, frame, min(a.steps, 10), flush, stream, crecs)
        conv = {"value": cnewton / (cms / 1e3), "unit": UNIT, "pcg": PCG_RULE.format(cap=a.converged_cap),
                "steps": min(a.steps, 10), "ms_per_step": cms / min(a.steps, 10), "residuals": _residual_summary(crecs)}

    # max over ranks of the time, sum of the work
    t_s = ms_total / 1e3
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
        solver_uses_rows = a.mode == "fused" and solver.uses_row_pcg()
        kind = solver.pcg_kind()
        pcg_kernel_name = {"cg1-res": "k_pcg_res (single-reduction slice-resident Jacobi-PCG)",
                           "cg1": "k_pcg_cg1 (single-reduction row-resident Jacobi-PCG)",
                           "rows": "k_pcg_rows (row-resident Jacobi-PCG)"}[kind] if solver_uses_rows else \
            ("k_pcg_fused (persistent Jacobi-PCG solve)" if a.mode == "fused" else "plain PCG kernels")
        # roofline of the dominant kernel: the persistent PCG solve (one launch per Newton iteration)
        pcg_ms, pcg_launches = prof["pcg"]
        nnz = cnt["nnz_material"] + 12 * int(np.mean([r["contact_pairs"] for r in recs]))
        it_per_launch = pcg / max(pcg_launches, 1)
        # algorithmic bytes of one PCG iteration: every matrix block once (36 B values + 4 B column), the
        # diagonal blocks (48 B/row) and the exchanged direction written and read once (32 B/row) when the row
        # state stays in registers (row-resident kernels); the CSR-vector kernel also streams r, z, p, q, x
        # (312 B/row in all)
        bytes_per_iter = 40.0 * nnz + (80.0 if solver_uses_rows else 312.0) * V
        bytes_per_launch = it_per_launch * bytes_per_iter + 160.0 * V
        achieved = bytes_per_launch / (pcg_ms / max(pcg_launches, 1) / 1e3) / 1e9
        peak, peak_kind = measured_peak()
        traffic = committed_traffic(pcg_kernel_name.split()[0])
        cpu = None
        if not a.no_cpu_baseline and world == 1:
            v_cpu, info = cpu_tube_steps(budget_s=15.0, warmup=0)
            cpu = {"value": v_cpu, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                   "sample": f"{info['steps']} time steps ({info['newton_iters']} Newton iterations, "
                             f"{info['seconds']:.1f} s) of the CPU restatement (oracle, OpenMP, all host cores) from "
                             "the same tube state"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_total / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" + ("+f64 reductions" if a.fp64 else ""), "data": "synthetic (seeded tube mesh)",
            "impl": "ours", "mode": a.mode, "pcg_kernel": kind, "traversal": a.traversal,
            "config": tube_config(frame),
            "parallelism": f"replicas x{world}" if world > 1 else "single scene",
            "e2e": None if a.e2e_steps == 0 else {
                "value": e2e_all / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 16 * V,
                "d2h_bytes_per_step": 2 * 16 * V, "steps": a.e2e_steps,
                "timing": "wall clock around lcs_newton_step_host (copies in, step, copies out, synchronise)"},
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
            "residuals": _residual_summary(recs),
            "first_iteration": {"vf": first["vf_candidates"], "ee": first["ee_candidates"],
                                "pairs": first["contact_pairs"]},
            "converged_1e-4": conv,
            "step_ms": {"min": min(p[0] for p in per_step), "median": statistics.median(p[0] for p in per_step),
                        "max": max(p[0] for p in per_step), "retries": sum(p[2] for p in per_step),
                        "host_ms_median": statistics.median(p[3] for p in per_step)},
            "phase_ms": {k: round(v[0], 3) for k, v in prof.items()},
            "iterations_of_a_step": [{k: (round(v, 6) if isinstance(v, float) else v) for k, v in r.items()}
                                     for r in recs[:per_step[0][1]]],
        }
        print(json.dumps(line), flush=True)
    del solver
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_c1(a):
    """C1 as configured: whole 10-step runs of the 64x64 cloth onto the pinned icosphere, from rest."""
    import numpy as np
    import torch
    from luisacomputesimulator_b200 import _capi, scenes
    from luisacomputesimulator_b200.newton import NewtonSolver
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    lib = _capi.load()
    _capi.check(lib.lcs_device_check(local), "device check")
    sc = scenes.cloth_on_sphere(n=64)
    solver = NewtonSolver(sc, single_reduction=True)
    stream = torch.cuda.current_stream()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
    x0, v0 = sc.x.copy(), np.zeros_like(sc.x)

    def run(records=None):
        solver.upload(x0, v0)
        solver.set_frame(0)
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        n = 0
        for _ in range(10):
            n += solver.step().newton_iters
            if records is not None:
                records += solver.iteration_log()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), n

    for _ in range(a.warmup):
        run()
    recs, ms, newton = [], 0.0, 0
    launches0 = lib.lcs_launch_count()
    with Clocks(local) as clk:
        for _ in range(a.steps):
            m, n = run(recs)
            ms += m
            newton += n
    launches = lib.lcs_launch_count() - launches0
    clocks = clk.summary()
    # end to end: host state in, ten steps through lcs_newton_step_host, state out each step
    V = sc.num_verts
    hx = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    hv = torch.empty((V, 4), dtype=torch.float32).pin_memory()
    e2e_s, e2e_n = 0.0, 0
    for k in range(min(a.steps, 5) + 1):
        hx.numpy()[:] = x0
        hv.numpy()[:] = v0
        solver.set_frame(0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n = 0
        for _ in range(10):
            n += solver.step_host(hx.numpy(), hv.numpy(), hx.numpy(), hv.numpy()).newton_iters
        el = time.perf_counter() - t0
        if k:
            e2e_s += el
            e2e_n += n
    if rank == 0:
        cpu = None
        if not a.no_cpu_baseline:
            v_cpu, info = cpu_c1_runs(budget_s=10.0, warmup=0)
            cpu = {"value": v_cpu, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                   "sample": f"{info['runs']} whole 10-step C1 runs ({info['newton_iters']} Newton iterations, "
                             f"{info['seconds']:.1f} s) of the CPU restatement (oracle, OpenMP, all host cores)"}
        line = {"metric": METRIC_C1, "value": newton / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded cloth grid, icosphere)", "impl": "ours",
                "config": c1_config(),
                "e2e": {"value": e2e_n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 10 * 2 * 16 * V,
                        "d2h_bytes_per_step": 10 * 2 * 16 * V, "steps": min(a.steps, 5),
                        "timing": "wall clock around ten lcs_newton_step_host calls"},
                "gpu_launches": int(launches), "cpu_baseline": cpu, "clocks": clocks, "newton_iters": newton,
                "residuals": _residual_summary(recs)}
        print(json.dumps(line), flush=True)


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
    q_vf, q_ee = batch.query_tuning()
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
                   "traversal_autotune": {"vf_threads_per_block": q_vf, "ee_threads_per_block": q_ee,
                                          "candidates": [64, 128, 256]},
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
    # twice (the batches sum in a fixed order, LCS_NEWTON_DETERMINISTIC: both deviations are 0)
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
        # batches admitted while another batch was still on the GPU (continuous batching at work)
        "batches_admitted_while_others_ran": sum(
            1 for b in server.log if any(o is not b and o["start"] < b["start"] < o["done"] for o in server.log)),
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
    elif a.workload == "c1":
        run_c1(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
