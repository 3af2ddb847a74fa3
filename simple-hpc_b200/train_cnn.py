"""Train the p' warm-start network on pairs the solver writes, then measure what it gains.

    python simple-hpc_b200/train_cnn.py --out unet.bin [--pairs 6000] [--steps 4000] [--eval 2048 4096]

1. Data: cavities with N uniform in [256, 1024] (multiples of 64) and Re log-uniform in [100, 3200],
   QUICK + 4th-order diffusion, gs_multicolour + mg, FP64. Each cavity advances with the reference's
   single V-cycle; at outer iterations sampled over the start-up transient (where the 4096^2 runs are
   measured) one outer iteration solves p' to 1e-10 (mg_mode = tolerance, sgpu_set_mg_mode) and the
   solver writes the pair (network input of the warm-start level, block mean of that converged p')
   through sgpu_cnn_sample.
2. Training: the U-Net (16/32/64/128 channels, 4 levels) with Adam on the GPU, batches of one grid
   size, cosine-decayed learning rate; a held-out 5% of the pairs gives the validation loss.
3. Evaluation (per --eval size, Re 2000, QUICK/4), the same K outer iterations each:
   - wall time per outer iteration: plain FP64 with the reference's settings (one V-cycle), mixed
     precision (one FP32 V-cycle), mixed precision with the network's guess as the V-cycle's start;
     their max / L2 relative error of u, v, p against the plain FP64 run;
   - what the guess gains the p' solve: V-cycles to ||b - A p'|| <= 1e-5 ||b|| (mg_mode =
     tolerance) from zero and from the guess, in FP64 and in mixed precision (FP32 V-cycles inside
     FP64 defect correction), with wall time per outer iteration and the error between the runs.

Prints one JSON line per stage; writes the weights to --out (sgpu_cnn_write format).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
import sgpu  # noqa: E402


def config(n: int, re: float, **kw) -> str:
    c = {"N_cells_x": n, "N_cells_y": n, "Re": repr(float(re)), "convection_scheme": "QUICK",
         "diffusion_order": 4, "momentum_solver": "gs_multicolour", "pressure_solver": "mg",
         "error_tolerance": 0, "maxit": 1000000}
    c.update(kw)
    return "".join(f"{k} = {v}\n" for k, v in c.items())


def generate(npairs: int, max_size: int, seed: int, per_cavity: int, max_iter: int) -> dict:
    rng = np.random.default_rng(seed)
    data: dict[tuple[int, int], list] = {}
    made, cavities = 0, 0
    t0 = time.time()
    while made < npairs:
        n = int(rng.integers(4, 17)) * 64
        re = float(np.exp(rng.uniform(np.log(100.0), np.log(3200.0))))
        # sample iterations log-uniformly over the transient
        its = np.unique(np.round(np.exp(rng.uniform(np.log(2), np.log(max_iter), per_cavity))).astype(int))
        p = sgpu.params_from_config(config(n, re))
        with sgpu.Solver(p) as s:
            it = 0
            for target in its:
                while it < target - 1:  # the reference's single V-cycle between samples
                    s.outer_iteration()
                    it += 1
                s.set_mg_mode(True, 1e-10, 300)  # the sampled iteration solves p' tightly
                s.outer_iteration()
                it += 1
                s.set_mg_mode(False)
                x, t, _ = s.cnn_sample(max_size)
                if np.isfinite(x).all() and np.isfinite(t).all():
                    # kept in FP16 on the host (the network's inputs are BF16 anyway): 50k pairs of up to
                    # 256^2 cells then take about 10 GB; batches are widened to FP32
                    data.setdefault(x.shape[:2], []).append((x.astype(np.float16), t.astype(np.float16)))
                    made += 1
                if made >= npairs:
                    break
        cavities += 1
    print(json.dumps({"stage": "generate", "pairs": made, "cavities": cavities,
                      "sizes": {f"{k[0]}x{k[1]}": len(v) for k, v in sorted(data.items())},
                      "seconds": round(time.time() - t0, 1)}), flush=True)
    return data


def split(data: dict, frac: float, rng) -> tuple[dict, dict]:
    tr, va = {}, {}
    for k, v in data.items():
        idx = rng.permutation(len(v))
        nv = max(1, int(len(v) * frac)) if len(v) > 4 else 0
        va[k] = [v[i] for i in idx[:nv]]
        tr[k] = [v[i] for i in idx[nv:]]
    return tr, {k: v for k, v in va.items() if v}


def batches(pool, batch, rng):
    idx = rng.integers(0, len(pool), min(batch, len(pool)))
    return (np.stack([pool[i][0] for i in idx]).astype(np.float32),
            np.stack([pool[i][1] for i in idx]).astype(np.float32))


def train(net, tr: dict, va: dict, steps: int, batch: int, lr: float, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    keys = sorted(tr)
    weights = np.array([len(tr[k]) for k in keys], float)
    weights /= weights.sum()
    t0 = time.time()
    hist = []
    for step in range(steps):
        k = keys[rng.choice(len(keys), p=weights)]
        x, t = batches(tr[k], batch, rng)
        cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / steps)) + 1e-5
        hist.append(net.train_step(x, t, float(cur)))
    secs = time.time() - t0
    vloss = []
    for k, pool in va.items():
        for i in range(0, len(pool), batch):
            x = np.stack([q[0] for q in pool[i:i + batch]]).astype(np.float32)
            t = np.stack([q[1] for q in pool[i:i + batch]]).astype(np.float32)
            vloss.append(float(np.mean((net.forward(x) - t) ** 2)) / max(float(np.mean(t ** 2)), 1e-30))
    out = {"stage": "train", "steps": steps, "batch": batch, "seconds": round(secs, 1),
           "loss_first_50": float(np.mean(hist[:50])), "loss_last_50": float(np.mean(hist[-50:])),
           "validation_relative_mse": float(np.mean(vloss)) if vloss else None,
           "params": net.num_params, "flops_per_pixel": net.flops_per_pixel}
    print(json.dumps(out), flush=True)
    return out


def evaluate(net, n: int, iters: int, max_size: int) -> dict:
    import torch

    def run(precision: str, warm: bool, tolerance_mode: bool):
        kw = {"precision": precision}
        if tolerance_mode:
            kw.update(mg_mode="tolerance", pressure_tolerance="1e-5", pressure_maxit=100)
        p = sgpu.params_from_config(config(n, 2000.0, **kw))
        with sgpu.Solver(p) as s:
            if warm:
                s.attach_cnn(net, max_size)
            stream = torch.cuda.ExternalStream(s.stream())
            cycles = []
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ms = 0.0
            for _ in range(iters):
                e0.record(stream)
                s.outer_iteration()
                e1.record(stream)
                e1.synchronize()
                ms += e0.elapsed_time(e1)
                cycles.append(s.last_solve_stats()["mg_vcycles"])
            fields = [s.download(f) for f in (0, 1, 2)]
            ws = s.warm_start_stats() if warm else None
        return {"ms_per_iteration": ms / iters, "vcycles_per_iteration": float(np.mean(cycles)),
                "fields": fields, "ws": ws}

    def errors(a, b):
        e = {}
        for fname, x, y in zip("uvp", a["fields"], b["fields"]):
            e[f"max_rel_{fname}"] = float(np.max(np.abs(x - y)) / np.max(np.abs(y)))
            e[f"l2_rel_{fname}"] = float(np.linalg.norm(x - y) / np.linalg.norm(y))
        return e

    runs = {
        "plain_fp64": run("fp64", False, False),        # the reference's settings: one V-cycle
        "mixed": run("mixed", False, False),            # FP32 inner solves, one V-cycle
        "mixed_cnn": run("mixed", True, False),         # one V-cycle from the network's guess
        "fp64_tol": run("fp64", False, True),           # V-cycles to ||r|| <= 1e-5 ||b|| from zero
        "fp64_tol_cnn": run("fp64", True, True),        # ... from the network's guess
        "mixed_tol": run("mixed", False, True),         # FP32 V-cycles in FP64 defect correction
        "mixed_tol_cnn": run("mixed", True, True),      # ... from the network's guess
    }
    out = {"stage": "evaluate", "N": n, "Re": 2000, "outer_iterations": iters}
    for k, r in runs.items():
        out[k] = {"ms_per_iteration": r["ms_per_iteration"], "vcycles_per_iteration": r["vcycles_per_iteration"]}
        if r["ws"]:
            out[k]["warm_starts"] = r["ws"]["used"]
            out[k]["discarded"] = r["ws"]["fallbacks"]
    out["mixed"].update(errors(runs["mixed"], runs["plain_fp64"]))
    out["mixed_cnn"].update(errors(runs["mixed_cnn"], runs["plain_fp64"]))
    out["fp64_tol_cnn"].update(errors(runs["fp64_tol_cnn"], runs["fp64_tol"]))
    out["mixed_tol_cnn"].update(errors(runs["mixed_tol_cnn"], runs["fp64_tol"]))
    out["mixed_tol"].update(errors(runs["mixed_tol"], runs["fp64_tol"]))
    out["vcycle_reduction_mixed_tol"] = 1.0 - (runs["mixed_tol_cnn"]["vcycles_per_iteration"] /
                                              runs["mixed_tol"]["vcycles_per_iteration"])
    out["time_ratio_mixed_tol_cnn_over_zero"] = (runs["mixed_tol_cnn"]["ms_per_iteration"] /
                                                 runs["mixed_tol"]["ms_per_iteration"])
    out["vcycle_reduction_fp64_tol"] = 1.0 - (runs["fp64_tol_cnn"]["vcycles_per_iteration"] /
                                             runs["fp64_tol"]["vcycles_per_iteration"])
    out["time_ratio_fp64_tol_cnn_over_zero"] = (runs["fp64_tol_cnn"]["ms_per_iteration"] /
                                                runs["fp64_tol"]["ms_per_iteration"])
    out["speedup_mixed_over_plain_fp64"] = runs["plain_fp64"]["ms_per_iteration"] / runs["mixed"]["ms_per_iteration"]
    out["speedup_mixed_cnn_over_plain_fp64"] = (runs["plain_fp64"]["ms_per_iteration"] /
                                                runs["mixed_cnn"]["ms_per_iteration"])
    print(json.dumps(out), flush=True)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--pairs", type=int, default=6000)
    ap.add_argument("--per-cavity", type=int, default=24)
    ap.add_argument("--max-iter", type=int, default=400)
    ap.add_argument("--max-size", type=int, default=256)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--eval", type=int, nargs="*", default=[2048, 4096])
    ap.add_argument("--eval-iters", type=int, default=20)
    ap.add_argument("--weights", help="skip training: evaluate this weights file")
    args = ap.parse_args()
    if args.weights:
        net = sgpu.Cnn(path=args.weights)
    else:
        data = generate(args.pairs, args.max_size, args.seed, args.per_cavity, args.max_iter)
        tr, va = split(data, 0.05, np.random.default_rng(args.seed + 1))
        net = sgpu.Cnn(16, 4, seed=args.seed & 0xFFFF)
        train(net, tr, va, args.steps, args.batch, args.lr, args.seed + 2)
        net.write(args.out)
    for n in args.eval:
        evaluate(net, n, args.eval_iters, args.max_size)
    net.close()


if __name__ == "__main__":
    main()
