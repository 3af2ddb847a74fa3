"""Benchmark: SIMPLE outer iterations of the lid-driven cavity on the B200 solver.

Workload (default): the 4096 x 4096 cavity at Re 1000, QUICK convection, 4th-order diffusion,
gs_multicolour momentum sweeps, multigrid pressure correction, tolerance 1e-5 — the configuration the
time-to-1e-5 metric is quoted on. Time to 1e-5 = (outer iterations to 1e-5) / (outer iterations per
second); the benchmark measures the second factor, a step being one SIMPLE outer iteration. Inputs
are the cavity's own initial state (u = v = p = 0, lid u = 1), so the data are synthetic by nature.

Output: one JSON line (rank 0). ``value`` is device-timed throughput with the fields resident in HBM;
``e2e`` is the same metric through the C ABI from pinned host buffers (initial fields uploaded, every
iteration's residuals read back for the stopping test, final fields downloaded); ``roofline`` covers
the dominant kernel (the streaming multicolour sweep); ``cpu_baseline`` times the reference's own
OpenMP code (oracle/_ref) on a bounded sample of the same workload.

--impl reference times the reference's CPU implementation of the same outer iteration (oracle/_ref,
OpenMP, all host threads; else the C restatement, one thread) on the same config and metric.
Multi-GPU (torchrun): one independent cavity per rank (the single-cavity path does not shard), value =
iterations of all ranks / max-over-ranks time.
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
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "simple-hpc_b200"))
sys.path.insert(0, str(REPO / "oracle"))

METRIC = "SIMPLE outer iterations per second, cavity 4096x4096 Re1000 QUICK/4 (time-to-1e-5 = iterations / this)"
UNIT = "outer_iterations/s"


def workload_config(n: int, precision: str | None) -> str:
    """Config text of the workload; precision None gives the reference's own keys only."""
    text = (f"N_cells_x = {n}\nN_cells_y = {n}\nRe = 1000\nconvection_scheme = QUICK\n"
            f"diffusion_order = 4\nmomentum_solver = gs_multicolour\npressure_solver = mg\n"
            f"error_tolerance = 1e-5\nmaxit = 60000\nbackend = gpu\n")
    return text + (f"precision = {precision}\n" if precision else "")


def workload_name(n: int, precision: str) -> str:
    return (f"cavity {n}x{n} Re1000 QUICK/4, gs_multicolour (4 sweeps) + mg V(2,2) omega 1.8, "
            f"{precision}, one outer iteration per step")


# ---- distributed plumbing (one process per GPU; NCCL only for the barrier and the max) ----

def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(x: float, world: int) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- clocks during the timed region ----

class Clocks:
    def __init__(self, index: int):
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks() -> dict:
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# ---- CPU baseline / reference arm ----

def reference_engine(text: str, n: int):
    """The reference's own OpenMP code when built (oracle/_ref), else the C restatement."""
    import oracle
    if oracle.ref_available():
        ref = oracle.Reference(text, (n + 5, n + 5))
        cores = oracle.ref_lib().ref_max_threads()
        return ref, "reference", cores
    import sgpu
    p = sgpu.params_from_config(text)
    return oracle.Oracle(p), "port", 1


def time_cpu_iterations(engine, iters: int) -> float:
    t0 = time.perf_counter()
    for _ in range(iters):
        engine.outer_iteration()
    return time.perf_counter() - t0


def run_reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    n = args.size
    text = workload_config(n, None)
    engine, kind, cores = reference_engine(text, n)
    for _ in range(args.warmup):
        engine.outer_iteration()
    secs = time_cpu_iterations(engine, args.steps)
    value = args.steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (cavity initial state)",
        "config": {"workload": workload_name(n, "fp64") + ", reference CPU OpenMP outer iteration",
                   "cells": n * n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{args.steps} outer iterations at {n}x{n} after {args.warmup} warm-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(n: int, seconds_budget: float) -> dict:
    text = workload_config(n, None)
    engine, kind, cores = reference_engine(text, n)
    engine.outer_iteration()  # first-touch / warm-up
    iters, secs = 0, 0.0
    while secs < seconds_budget and iters < 50:
        secs += time_cpu_iterations(engine, 1)
        iters += 1
    engine.close()
    return {"value": iters / secs, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{iters} outer iterations of the same {n}x{n} workload after 1 warm-up "
                      f"({secs:.1f} s)"}


# ---- GPU arm ----

def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3

    rank, world, local = dist_init()
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        barrier(world)
        return

    import torch
    import sgpu

    torch.cuda.set_device(local)
    n = args.size
    p = sgpu.params_from_config(workload_config(n, args.precision))
    solver = sgpu.Solver(p)
    stream = torch.cuda.ExternalStream(solver.stream())

    # warm-up (untimed)
    for _ in range(args.warmup):
        solver.outer_iteration()

    # ---- device-timed region: K outer iterations, fields resident in HBM ----
    solver.set_profiling(True)
    ph0 = solver.phase_seconds()
    launches0 = sgpu.launch_count()
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res, log = solver.run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    launches = sgpu.launch_count() - launches0
    ph1 = solver.phase_seconds()
    solver.set_profiling(False)
    secs = e0.elapsed_time(e1) * 1e-3
    secs_max = allmax(secs, world)
    iters = res.iterations
    value = world * iters / secs_max

    # ---- roofline of the dominant kernel (the streaming sweep, 2 x maxit_inner launches) ----
    sweep_s = (ph1["sweep_u"] - ph0["sweep_u"]) + (ph1["sweep_v"] - ph0["sweep_v"])
    sweep_launches = iters * (p.maxit_inner_u + p.maxit_inner_v)
    cells = p.nrows * p.ncols
    bytes_per_launch = 5 * 8 * cells  # read x_in, frozen x, other velocity, p; write x_out
    per_launch_s = sweep_s / max(sweep_launches, 1)
    peaks = measured_peaks()
    achieved = bytes_per_launch / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    traffic = None
    prof = REPO / "profiles" / "sweep_traffic.json"
    if prof.exists():
        t = json.loads(prof.read_text())
        traffic = t.get("bytes_per_cell", 0) * cells if t.get("bytes_per_cell") else None

    phases_ms = {k: 1e3 * (ph1[k] - ph0[k]) / max(iters, 1) for k in ph1 if k != "output"}

    # ---- end to end through the C ABI from pinned host memory ----
    e2e = None
    if rank == 0 or world > 1:
        shape = (p.nrows, p.ncols)
        pinned = [torch.zeros(shape, dtype=torch.float64).pin_memory() for _ in range(3)]
        hu, hv, hp = (t.numpy() for t in pinned)
        solver2 = sgpu.Solver(p)  # allocation outside the timed region
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver2.upload(sgpu.F_U, hu)
        solver2.upload(sgpu.F_V, hv)
        solver2.upload(sgpu.F_P, hp)
        r2, _ = solver2.run(args.steps)
        out_u, out_v, out_p = (solver2.download(f) for f in (sgpu.F_U, sgpu.F_V, sgpu.F_P))
        t_e2e = time.perf_counter() - t0
        solver2.close()
        t_e2e = allmax(t_e2e, world)
        fb = 8 * p.nrows * p.ncols
        e2e = {"value": world * r2.iterations / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": 3 * fb / r2.iterations,
               "d2h_bytes_per_step": 24 + 3 * fb / r2.iterations}
        del out_u, out_v, out_p

    solver.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(n, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": iters,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs_max / max(iters, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64+f32",
            "data": "synthetic (cavity initial state u=v=p=0, lid u=1)",
            "config": {"workload": workload_name(n, args.precision), "cells": n * n,
                       "grid": f"{n}x{n}", "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (each field 134 MB at 4096^2; ~30 fields per step)",
                       "converged_in_timed_region": bool(res.converged)},
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "roofline": {"bound": "hbm", "kernel": "k_mom_stream (one multicolour sweep)",
                         "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                         "peak_source": peaks["source"],
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "avg_launch_ms": per_launch_s * 1e3},
            "phases_ms_per_step": phases_ms,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
