"""Benchmark: SIMPLE outer iterations of the lid-driven cavity on the B200 solver.

Workload (default): the 4096 x 4096 cavity at Re 1000, QUICK convection, 4th-order diffusion,
gs_multicolour momentum sweeps, multigrid pressure correction, tolerance 1e-5 — the configuration the
time-to-1e-5 metric is quoted on. Time to 1e-5 = (outer iterations to 1e-5) / (outer iterations per
second); the benchmark measures the second factor, a step being one SIMPLE outer iteration. Inputs
are the cavity's own initial state (u = v = p = 0, lid u = 1), so the data are synthetic by nature.

The headline arm is the mixed-precision solve (FP32 inner solves inside FP64 defect correction,
precision = mixed); the plain FP64 GPU solve (bit-identical to the reference) is timed in the same
run on the same K steps, and the line reports both and their ratio.

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
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "simple-hpc_b200"))
sys.path.insert(0, str(REPO / "oracle"))

METRIC = ("SIMPLE outer iterations per second, cavity 4096x4096 Re1000 QUICK/4 gs_multicolour+mg "
          "(time-to-1e-5 = iterations / this)")
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
    """Max over ranks (the job's time is its slowest rank's)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- clocks during the timed region ----

class Clocks:
    """SM clock and throttle reasons of this process's GPU, sampled every 10 ms by an NVML thread
    while the timed region runs (read-only queries). The GPU is found by its UUID, so the sample is
    of the same device under CUDA_VISIBLE_DEVICES."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int, period: float = 0.01):
        import threading
        self.sm, self.smax, self.reasons, self.err = [], [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self.nv = pynvml
            self.smax.append(float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)))
        except Exception as e:  # no NVML: the line says so
            self.h, self.err = None, f"nvml unavailable: {type(e).__name__}: {e}"
            return
        self.period = period
        self._sample()
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _sample(self):
        nv = self.nv
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        for name, bit in self.REASONS.items():
            if mask & bit:
                self.reasons.add(name)

    def _run(self):
        while not self._stop.wait(self.period):
            try:
                self._sample()
            except Exception as e:
                self.err = f"{type(e).__name__}: {e}"
                return

    def stop(self) -> dict:
        if self.h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": [self.err]}
        self._stop.set()
        self.t.join(timeout=2)
        self._sample()
        out = {"sm_mhz": statistics.median(self.sm), "sm_min_mhz": min(self.sm),
               "sm_max_mhz": max(self.smax), "samples": len(self.sm), "reasons": sorted(self.reasons),
               "source": "NVML, every 10 ms during the timed region"}
        if self.err:
            out["error"] = self.err
        return out


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

def measure(sgpu, torch, n: int, precision: str, steps: int, warmup: int, world: int, local: int,
            clocks: bool) -> dict:
    """Device-timed K outer iterations (fields resident in HBM) through sgpu_run, which replays the
    captured iteration graph with the stopping test on the device; then a profiled pass of the
    same iterations for the per-phase and sweep-kernel times (per-phase events need host-issued
    launches, so that pass is not the timed one)."""
    p = sgpu.params_from_config(workload_config(n, precision))
    solver = sgpu.Solver(p)
    stream = torch.cuda.ExternalStream(solver.stream())
    solver.run(warmup)  # warm-up; also captures the iteration graph
    launches0 = sgpu.launch_count()
    clk = Clocks(local) if clocks else None
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res, _ = solver.run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk_info = clk.stop() if clk else None
    launches = sgpu.launch_count() - launches0
    # profiled pass (host-issued launches with per-phase events)
    solver.set_profiling(True)
    ph0 = solver.phase_seconds()
    sw0 = solver.sweep_seconds()
    prof = solver.run(steps)[0].iterations
    ph1 = solver.phase_seconds()
    sw1 = solver.sweep_seconds()
    # final u, v, p (after warmup + 2 x steps iterations, the same count in every arm)
    fields = [solver.download(f) for f in (sgpu.F_U, sgpu.F_V, sgpu.F_P)]
    solver.close()
    secs = allmax(e0.elapsed_time(e1) * 1e-3, world)
    iters = res.iterations
    return {"p": p, "iters": iters, "secs": secs, "value": world * iters / secs,
            "ms_per_step": 1e3 * secs / max(iters, 1), "launches": launches, "clocks": clk_info,
            "phases": {k: (ph1[k] - ph0[k]) * iters / max(prof, 1) for k in ph1 if k != "output"},
            "sweep_s": sw1[0] - sw0[0], "sweep_launches": sw1[1] - sw0[1],
            "converged": bool(res.converged), "fields": fields,
            "iterations_total": warmup + iters + prof}


def field_errors(a_fields, b_fields) -> dict:
    """max |a - b| / max |b| and ||a - b|| / ||b|| of u, v, p (b: the plain FP64 run)."""
    import numpy as np
    out = {}
    for name, a, b in zip("uvp", a_fields, b_fields):
        out[name] = {"max_rel": float(np.max(np.abs(a - b)) / np.max(np.abs(b))),
                     "l2_rel": float(np.linalg.norm(a - b) / np.linalg.norm(b))}
    return out


def e2e_measure(sgpu, torch, p, steps: int, world: int) -> dict:
    """The same K iterations through the C ABI from pinned host buffers, copies included."""
    shape = (p.nrows, p.ncols)
    pinned = [torch.zeros(shape, dtype=torch.float64).pin_memory() for _ in range(6)]
    hu, hv, hp, ou, ov, op = (t.numpy() for t in pinned)
    solver = sgpu.Solver(p)  # allocation outside the timed region
    solver.run(2)            # and the capture of the iteration graph
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solver.upload(sgpu.F_U, hu)
    solver.upload(sgpu.F_V, hv)
    solver.upload(sgpu.F_P, hp)
    res, _ = solver.run(steps)
    for f, out in ((sgpu.F_U, ou), (sgpu.F_V, ov), (sgpu.F_P, op)):
        solver.download(f, out)
    t = allmax(time.perf_counter() - t0, world)
    solver.close()
    fb = 8 * p.nrows * p.ncols
    return {"value": world * res.iterations / t, "unit": UNIT,
            "h2d_bytes_per_step": 3 * fb / res.iterations,
            "d2h_bytes_per_step": 32 + 3 * fb / res.iterations}


# ---- the reference's own GPU backend on the same B200 ----

def reference_gpu_bar(sgpu, torch, sizes, steps: int, warmup: int) -> dict | None:
    """simple-hpc's HipSolver (solver_hip.hip built as CUDA for sm_100a by oracle/Makefile), which
    supports gs_multicolour + gs_redblack only, against this repository's FP64 solver with the same
    solvers on the same iterations. The reference is timed by wall clock around its
    outer_iteration (a device synchronisation per phase, as it runs); ours by CUDA events around
    sgpu_run. Fields are compared bit for bit after the same iteration count."""
    import numpy as np
    import oracle
    if not oracle.refgpu_available():
        return None
    out = {}
    for n in sizes:
        text = workload_config(n, None).replace("pressure_solver = mg", "pressure_solver = gs_redblack")
        shape = (n + 5, n + 5)
        ref = oracle.ReferenceGpu(text, shape)
        ref.iterations(warmup)
        rsecs, _ = ref.iterations(steps)
        theirs = [ref.get(f) for f in (0, 1, 2)]
        ref.close()
        p = sgpu.params_from_config(text)
        s = sgpu.Solver(p)
        stream = torch.cuda.ExternalStream(s.stream())
        s.run(warmup)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res, _ = s.run(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        osecs = e0.elapsed_time(e1) * 1e-3
        ours = [s.download(f) for f in (0, 1, 2)]
        s.close()
        same = all(np.array_equal(a.view(np.uint64), b.view(np.uint64)) for a, b in zip(ours, theirs))
        out[f"{n}x{n}"] = {"reference_ms_per_iteration": 1e3 * rsecs / steps,
                           "ours_ms_per_iteration": 1e3 * osecs / res.iterations,
                           "speedup": (rsecs / steps) / (osecs / res.iterations),
                           "fields_bit_identical": same}
    return {"solvers": "gs_multicolour + gs_redblack (the only pair the reference GPU backend supports), "
                       "QUICK/4, Re 1000, FP64",
            "reference": "simple-hpc src/hip/solver_hip.hip, nvcc -x cu -DSIMPLE_CUDA --fmad=false, sm_100a",
            "steps": steps, "warmup": warmup, "sizes": out}


# ---- the metric itself where it is reachable: time to the residual tolerance ----

CONVERGE_METRIC = ("wall time to error_tolerance 1e-5 (absolute residuals, the reference's stopping rule), "
                   "cavity NxN Re1000 QUICK/4 gs_multicolour+mg")
WEIGHTS = REPO / "simple-hpc_b200" / "weights" / "unet16_l4_cavity.bin"


def converge_config(n: int, precision: str | None, warm: bool, maxit: int) -> str:
    text = workload_config(n, precision).replace("maxit = 60000", f"maxit = {maxit}")
    if warm:
        text += f"warm_start = cnn\ncnn_weights = {WEIGHTS}\n"
    return text


def refgpu_arms(sgpu, torch, n: int, maxit: int, world: int, out: dict) -> None:
    """The pair the reference's GPU backend supports, gs_multicolour + gs_redblack, to 1e-5: the
    reference's own HipSolver under its own run_outer_loop (wall time, a device synchronisation per
    phase as it runs), and this repository's FP64 solver on the same settings."""
    import oracle
    if not oracle.refgpu_available():
        return
    text = converge_config(n, None, False, maxit).replace("pressure_solver = mg", "pressure_solver = gs_redblack")
    ref = oracle.ReferenceGpu(text, (n + 5, n + 5))
    its, conv, secs = ref.run()
    theirs = [ref.get(f) for f in (0, 1, 2)]
    ref.close()
    p = sgpu.params_from_config(text)
    with sgpu.Solver(sgpu.params_from_config(text.replace(f"maxit = {maxit}", "maxit = 5"))) as w:
        w.run(3)
    s = sgpu.Solver(p)
    stream = torch.cuda.ExternalStream(s.stream())
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res, _ = s.run(p.maxit)
    e1.record(stream)
    torch.cuda.synchronize()
    osecs = allmax(e0.elapsed_time(e1) * 1e-3, world)
    ours = [s.download(f) for f in (0, 1, 2)]
    s.close()
    import numpy as np
    same = all(np.array_equal(a.view(np.uint64), b.view(np.uint64)) for a, b in zip(ours, theirs))
    out["reference_gpu_rb"] = {"seconds": secs, "iterations": its, "converged": conv,
                               "ms_per_iteration": 1e3 * secs / max(its, 1),
                               "note": "simple-hpc's own GPU backend (solver_hip.hip as CUDA, sm_100a) under "
                                       "its run_outer_loop, gs_multicolour + gs_redblack",
                               "fields": theirs}
    out["fp64_rb"] = {"seconds": osecs, "iterations": res.iterations, "converged": bool(res.converged),
                      "ms_per_iteration": 1e3 * osecs / max(res.iterations, 1),
                      "speedup_vs_reference_gpu": secs / osecs, "fields_bit_identical_to_reference_gpu": same,
                      "fields": ours}


def run_converge_workload(args, rank: int, world: int, local: int) -> None:
    """Each size is solved to error_tolerance 1e-5 by: the plain FP64 method (the reference's
    settings, bit-identical to it), mixed precision, and mixed precision with the learned warm start
    (the network's guess as the start of each p' solve, judged after its first V-cycle). A fresh
    solver runs each arm from the cavity's initial state; its time is the device time of sgpu_run
    (CUDA events around it on the solver's stream) plus, separately, the host's wall time. Errors are
    of u, v, p against the FP64 arm. The 128^2 case sits beside the reference's published Ghia-size
    run: 128^2 Re 1000 to 1e-5, 5919 iterations in 1.79 s on an H100 (docs/RESULTS.md:335)."""
    import numpy as np
    import torch
    import sgpu
    torch.cuda.set_device(local)
    arms = [("fp64", None, False), ("mixed", "mixed", False)]
    if WEIGHTS.exists() and not args.no_cnn:
        arms.append(("mixed_cnn", "mixed", True))
    rows = []
    for n in args.converge_sizes:
        # warm-up: module load, graph capture paths, on a separate solver of the same size
        for name, prec, warm in arms:
            with sgpu.Solver(sgpu.params_from_config(converge_config(n, prec, warm, 5))) as w:
                w.run(3)
        out = {}
        for name, prec, warm in arms:
            p = sgpu.params_from_config(converge_config(n, prec, warm, args.converge_maxit))
            s = sgpu.Solver(p)
            stream = torch.cuda.ExternalStream(s.stream())
            barrier(world)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            res, log = s.run(p.maxit)
            e1.record(stream)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            secs = allmax(e0.elapsed_time(e1) * 1e-3, world)
            fields = [s.download(f) for f in (sgpu.F_U, sgpu.F_V, sgpu.F_P)]
            ws = s.warm_start_stats() if warm else None
            s.close()
            out[name] = {"seconds": secs, "wall_seconds": wall, "iterations": res.iterations,
                         "converged": bool(res.converged),
                         "ms_per_iteration": 1e3 * secs / max(res.iterations, 1),
                         "vcycles_per_iteration": res.mg_vcycles / max(res.iterations, 1),
                         "final_residuals": [float(x) for x in log[-1, 1:]] if log.shape[0] else None,
                         "fields": fields}
            if ws is not None:
                out[name]["warm_start"] = ws
        if n <= args.converge_refgpu_max and not args.no_reference_gpu:
            refgpu_arms(sgpu, torch, n, args.converge_maxit, world, out)
        ref = out["fp64"]["fields"]
        for name in out:
            f = out[name].pop("fields")
            if name in ("mixed", "mixed_cnn"):
                out[name]["errors_vs_fp64"] = field_errors(f, ref)
                out[name]["speedup_vs_fp64"] = out["fp64"]["seconds"] / out[name]["seconds"]
        rows.append({"N": n, "arms": out})
    if rank == 0:
        last = rows[-1]["arms"]
        head = "mixed_cnn" if "mixed_cnn" in last else "mixed"
        line = {
            "metric": CONVERGE_METRIC + f" (headline: {head} at {rows[-1]['N']}^2)",
            "value": last[head]["seconds"], "unit": "s", "n_gpus": world, "steps": 1, "warmup": 1,
            "ms_per_step": 1e3 * last[head]["seconds"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (outer) + f32 (inner solves)",
            "data": "synthetic (cavity initial state u=v=p=0, lid u=1)",
            "config": {"workload": "cavities to 1e-5: " + ", ".join(f"{r['N']}^2" for r in rows) +
                                   "; arms fp64 (reference method), mixed, mixed + learned warm start",
                       "parallelism": f"replicas x{world}", "l2": "whole solve timed (many iterations)"},
            "sizes": rows,
            "reference_published": {"case": "128^2 Re1000 QUICK/4 gs_multicolour+gs_redblack to 1e-5 (Ghia run)",
                                    "iterations": 5919, "seconds": 1.79, "hardware": "H100 80GB",
                                    "source": "simple-hpc docs/RESULTS.md:335"},
        }
        print(json.dumps(line), flush=True)


# ---- batched workload: many cavities of uneven size and Re in one graph launch ----

BATCH_SIZES = (64, 96, 128, 192, 256, 384, 512)
BATCH_METRIC = ("cavities solved to 1e-5 per second: N uniform in {64,96,128,192,256,384,512}, Re "
                "log-uniform in [100, 5000], QUICK + 2nd-order diffusion, mixed-precision mg, one graph launch")


def batch_manifest(count: int, seed: int) -> list[tuple[int, float]]:
    import numpy as np
    rng = np.random.default_rng(seed)
    ns = rng.choice(BATCH_SIZES, count)
    res = np.exp(rng.uniform(np.log(100.0), np.log(5000.0), count))
    return [(int(n), float(r)) for n, r in zip(ns, res)]


def batch_config(n: int, re: float, precision: str | None, maxit: int) -> str:
    text = (f"N_cells_x = {n}\nN_cells_y = {n}\nRe = {re!r}\nconvection_scheme = QUICK\n"
            f"diffusion_order = 2\nmomentum_solver = gs_multicolour\npressure_solver = mg\n"
            f"error_tolerance = 1e-5\nmaxit = {maxit}\nbackend = gpu\n")
    return text + (f"precision = {precision}\n" if precision else "")


def batch_shard(manifest, world: int, rank: int):
    """Size-balanced partition (cost ~ N^3: cells x iterations), no collective needed."""
    load = [0.0] * world
    mine = []
    for idx in sorted(range(len(manifest)), key=lambda i: -manifest[i][0]):
        r = min(range(world), key=lambda k: load[k])
        load[r] += float(manifest[idx][0]) ** 3
        if r == rank:
            mine.append(idx)
    return sorted(mine)


def run_batch_workload(args, rank: int, world: int, local: int) -> None:
    import numpy as np
    import torch
    import sgpu
    torch.cuda.set_device(local)
    manifest = batch_manifest(args.cavities, args.seed)
    mine = batch_shard(manifest, world, rank)
    params = [sgpu.params_from_config(batch_config(*manifest[i], "mixed", args.batch_maxit)) for i in mine]
    # warm-up: short runs of a separate batch of the same cavities (module load, graph paths)
    with sgpu.Batch(params) as wb:
        wb.autotune()
        for _ in range(args.warmup):
            wb.run(2)
    t_wall0 = time.perf_counter()
    b = sgpu.Batch(params)
    chosen = b.autotune()
    barrier(world)
    torch.cuda.synchronize()
    secs = b.run(args.batch_maxit)
    torch.cuda.synchronize()
    barrier(world)
    r = b.results()
    fields = {i: [b.download(k, f) for f in (0, 1, 2)] for k, i in enumerate(mine)}
    wall = time.perf_counter() - t_wall0
    secs_max = allmax(secs, world)
    wall_max = allmax(wall, world)
    converged = int(r["converged"].sum())
    its = {i: int(r["iterations"][k]) for k, i in enumerate(mine)}
    b.close()
    out_bytes = sum(3 * 8 * p.nrows * p.ncols for p in params)
    # per-cavity error against individual FP64 runs: the first batch_check cavities of each size
    errs = []
    check = []
    for n_ in BATCH_SIZES:
        check += [i for i in mine if manifest[i][0] == n_][:args.batch_check]
    for i in check:
        p64 = sgpu.params_from_config(batch_config(*manifest[i], None, args.batch_maxit))
        with sgpu.Solver(p64) as s:
            res, _ = s.run(args.batch_maxit)
            ref = [s.download(f) for f in (0, 1, 2)]
        e = {"cavity": i, "N": manifest[i][0], "Re": round(manifest[i][1], 1), "iterations_fp64": res.iterations,
             "iterations_batch": its[i]}
        for name, a, x in zip("uvp", fields[i], ref):
            e[f"max_rel_{name}"] = float(np.max(np.abs(a - x)) / np.max(np.abs(x)))
            e[f"l2_rel_{name}"] = float(np.linalg.norm(a - x) / np.linalg.norm(x))
        errs.append(e)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = batch_cpu_estimate(manifest, its, args.cpu_seconds)
    if rank == 0:
        line = {
            "metric": BATCH_METRIC, "value": len(manifest) / secs_max, "unit": "cavities/s",
            "n_gpus": world, "steps": 1, "warmup": args.warmup, "ms_per_step": 1e3 * secs_max,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64 (outer) + f32 (inner solves)",
            "data": f"synthetic (seeded manifest, seed {args.seed}; cavity initial state)",
            "config": {"workload": f"{len(manifest)} cavities, batch to 1e-5 (maxit {args.batch_maxit}), "
                                   "one CUDA graph launch per rank (WHILE over per-cavity IF branches)",
                       "cavities": len(manifest), "sizes": list(BATCH_SIZES),
                       "parallelism": f"size-balanced shard x{world}", "step": "the whole batched solve",
                       "autotuned_row_segments": sorted(set(chosen))},
            "converged": converged if world == 1 else None,
            "iterations": {"min": min(its.values()), "max": max(its.values()),
                           "sum": sum(its.values())} if world == 1 else None,
            "e2e": {"value": len(manifest) / wall_max, "unit": "cavities/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": out_bytes,
                    "note": "batch creation, autotune, graph build, launch and download of every u, v, p"},
            "gpu_launches": 1,
            "errors_vs_fp64_single_runs": errs,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)


def batch_cpu_estimate(manifest, its: dict, budget: float) -> dict:
    """The reference's OpenMP outer iteration timed per distinct N (bounded sample), times the
    batch's iteration counts: the CPU time the reference would need for the same cavities."""
    per_n = {}
    spent = 0.0
    cores, kind = 1, "port"
    for n in sorted({m[0] for m in manifest}):
        engine, kind, cores = reference_engine(batch_config(n, 1000.0, None, 10), n)
        engine.outer_iteration()
        k, secs = 0, 0.0
        while k < 3 and (k == 0 or spent + secs < budget):
            secs += time_cpu_iterations(engine, 1)
            k += 1
        engine.close()
        spent += secs
        per_n[n] = secs / k
    est = sum(its[i] * per_n[manifest[i][0]] for i in its)
    return {"value": len(manifest) / est, "unit": "cavities/s", "cores": cores, "kind": kind,
            "sample": "outer iterations timed per N ({}); estimate = sum over cavities of the batch's "
                      "iteration count x that time ({:.0f} s)".format(
                          ", ".join(f"{n}: {1e3 * t:.2f} ms" for n, t in per_n.items()), est)}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-arm", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--workload", default="cavity", choices=["cavity", "batch", "converge"])
    ap.add_argument("--converge-sizes", type=int, nargs="+", default=[128, 256, 512])
    ap.add_argument("--converge-maxit", type=int, default=400000)
    ap.add_argument("--no-cnn", action="store_true")
    ap.add_argument("--converge-refgpu-max", type=int, default=256)
    ap.add_argument("--cavities", type=int, default=256)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--batch-maxit", type=int, default=60000)
    ap.add_argument("--batch-check", type=int, default=2, help="cavities per size checked against single FP64 runs")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3

    rank, world, local = dist_init()
    if args.impl == "reference" and args.workload == "converge":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "converge workload: the reference CPU needs "
                              "16 500 iterations (132 s) at 256^2 and 61 109 (1971 s) at 512^2 on 8 threads; "
                              "its published 128^2 GPU run is in the line's reference_published"}), flush=True)
        barrier(world)
        return
    if args.impl == "reference" and args.workload == "batch":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched mode and "
                              "needs hours per 512^2 cavity; the batch line's cpu_baseline times its outer "
                              "iteration per size and scales by the batch's iteration counts"}), flush=True)
        barrier(world)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        barrier(world)
        return

    if args.workload == "converge":
        run_converge_workload(args, rank, world, local)
        barrier(world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "batch":
        run_batch_workload(args, rank, world, local)
        barrier(world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    import sgpu

    torch.cuda.set_device(local)
    n = args.size
    head = measure(sgpu, torch, n, args.precision, args.steps, args.warmup, world, local, True)
    p = head["p"]
    plain = None
    if args.precision != "fp64" and not args.no_fp64_arm:
        plain = measure(sgpu, torch, n, "fp64", args.steps, args.warmup, world, local, False)

    # Roofline of the dominant kernel: the streaming sweep (2 x maxit_inner launches per step), timed
    # alone by the solver's own events around its back-to-back launches.
    ph = head["phases"]
    sweep_s, sweep_launches = head["sweep_s"], head["sweep_launches"]
    cells = (p.NX - 1) * p.NY  # cells one sweep updates: u NX x (NY-1), v (NX-1) x NY (square grid)
    if args.precision == "mixed":
        kernel = "k_corr_stream (one FP32 multicolour correction sweep)"
        bytes_per_cell = 40 + 4 + 4  # record (near links, far links, 1/AP and R) read, e_in read, e_out written
    else:
        kernel = "k_mom_stream (one FP64 multicolour sweep)"
        bytes_per_cell = 5 * 8  # x_in, frozen x, other velocity, p read; x_out written
    bytes_per_launch = bytes_per_cell * cells
    per_launch_s = sweep_s / max(sweep_launches, 1)
    peaks = measured_peaks()
    achieved = bytes_per_launch / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    traffic = None
    prof = REPO / "profiles" / "sweep_traffic.json"
    if prof.exists():
        t = json.loads(prof.read_text()).get(args.precision, {})
        if t.get("bytes_per_cell"):
            traffic = t["bytes_per_cell"] * cells

    e2e = e2e_measure(sgpu, torch, p, args.steps, world)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_bar(sgpu, torch, (2048, n), 10, 2)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(n, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": head["iters"], "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64 (outer) + f32 (inner solves)",
            "data": "synthetic (cavity initial state u=v=p=0, lid u=1)",
            "config": {"workload": workload_name(n, args.precision), "cells": n * n,
                       "grid": f"{n}x{n}", "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (each FP64 field 135 MB at 4096^2; ~40 arrays per step)",
                       "converged_in_timed_region": head["converged"]},
            "plain_fp64": None if plain is None else {
                "value": plain["value"], "ms_per_step": plain["ms_per_step"],
                "note": "bit-identical to the reference (tests/test_gpu_scale.py checks 4096^2 x 3 and "
                        "1024^2 x 50 iterations against the reference's own build); same K steps, same run"},
            "errors_vs_fp64": None if plain is None else {
                "after_iterations": head["iterations_total"],
                "fields": field_errors(head["fields"], plain["fields"]),
                "note": "mixed arm against the plain FP64 arm of this run, same iteration count"},
            "timing": "sgpu_run replays the captured outer-iteration graph (WHILE node, device-side "
                      "stopping test); per-phase times come from a separate profiled pass",
            "mixed_vs_fp64": None if plain is None else head["value"] / plain["value"],
            "e2e": e2e,
            "gpu_launches": head["launches"],
            "clocks": head["clocks"],
            "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "traffic": traffic, "peak_source": peaks["source"],
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "avg_launch_ms": per_launch_s * 1e3},
            "phases_ms_per_step": {k: 1e3 * v / max(head["iters"], 1) for k, v in ph.items()},
            "reference_gpu": ref_gpu,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
