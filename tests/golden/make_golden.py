"""Regenerate the golden fixtures in this folder from the reference (run where the reference exists).

Two kinds of fixture, both float64 .npz files:

* ``snapshot_<name>.npz`` — the reference's committed regression snapshots
  (tests/snapshots/short_16 and converged_32x40 in simple-hpc: u, v, p and alog CSVs written with
  %.18e, which round-trips every double exactly) together with the config they were made with
  (configs/snapshot/<name>.cfg). Both are gs_lex / gs_lex runs on the CPU.
* ``run_<tag>.npz`` — runs of the reference's own C++ sources, built in place into
  oracle/_ref/libsimpleref.so (oracle/Makefile), for the GPU backend's solver combinations:
  final u, v, p and the residual log.

Usage:  python tests/golden/make_golden.py [REFERENCE_DIR] [TAG ...]
(with tags, only those run fixtures are written)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "oracle"))

import oracle  # noqa: E402

# (tag, base config, overrides, iterations)
RUNS = [
    ("mc_rb_quick4_32x40", "converged_32x40",
     {"momentum_solver": "gs_multicolour", "pressure_solver": "gs_redblack",
      "error_tolerance": "0", "maxit": "40"}, 40),
    ("mc_mg_quick4_32x40", "converged_32x40",
     {"momentum_solver": "gs_multicolour", "pressure_solver": "mg",
      "error_tolerance": "0", "maxit": "40"}, 40),
    ("mc_cg_uds2_32x40", "converged_32x40",
     {"momentum_solver": "gs_multicolour", "pressure_solver": "cg", "convection_scheme": "UDS",
      "diffusion_order": "2", "error_tolerance": "0", "maxit": "25"}, 25),
    ("jac_jac_quick4_16", "short_16",
     {"momentum_solver": "jacobi", "pressure_solver": "jacobi", "maxit": "10"}, 10),
    # The plain-method CPU configuration: 32x32, Re 100, QUICK + 2nd-order diffusion,
    # gs_multicolour + mg, tolerance 1e-5, run to convergence.
    ("cavity32_re100_mc_mg", None,
     {"N_cells_x": "32", "N_cells_y": "32", "Re": "100", "convection_scheme": "QUICK",
      "diffusion_order": "2", "momentum_solver": "gs_multicolour", "pressure_solver": "mg",
      "error_tolerance": "1e-5", "maxit": "60000"}, 60000),
    # The converged_32x40 snapshot's own stopping rule (residual_normalisation = running_max,
    # tolerance 1e-4), run to convergence with the GPU backend's solver combinations.
    ("runmax_mc_mg_32x40", "converged_32x40",
     {"momentum_solver": "gs_multicolour", "pressure_solver": "mg"}, 15000),
    ("runmax_mc_rb_32x40", "converged_32x40",
     {"momentum_solver": "gs_multicolour", "pressure_solver": "gs_redblack"}, 15000),
]


def config_text(ref: Path, base: str | None, overrides: dict) -> str:
    lines = []
    if base:
        lines = (ref / "configs" / "snapshot" / f"{base}.cfg").read_text().splitlines()
        lines = [ln for ln in lines if ln.split("#")[0].split("=")[0].strip() not in overrides]
    return "\n".join(lines + [f"{k} = {v}" for k, v in overrides.items()]) + "\n"


def parse_cfg(text: str) -> dict:
    out = {}
    for ln in text.splitlines():
        ln = ln.split("#")[0].strip()
        if ln:
            k, v = ln.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def main(ref: Path, tags: list[str]) -> None:
    for name in ("short_16", "converged_32x40"):
        if tags:
            break
        d = ref / "tests" / "snapshots" / name
        cfg = (ref / "configs" / "snapshot" / f"{name}.cfg").read_text()
        arrs = {k: np.loadtxt(d / f"{k}.csv", delimiter=",", dtype=np.float64) for k in ("u", "v", "p")}
        alog = np.loadtxt(d / "alog.csv", delimiter=",", skiprows=1, dtype=np.float64, ndmin=2)
        np.savez_compressed(HERE / f"snapshot_{name}.npz", **arrs, alog=alog,
                            config=json.dumps(parse_cfg(cfg)))
        print(f"snapshot_{name}.npz", {k: v.shape for k, v in arrs.items()}, alog.shape)

    for tag, base, ov, iters in RUNS:
        if tags and tag not in tags:
            continue
        text = config_text(ref, base, ov)
        cfg = parse_cfg(text)
        nx, ny = int(cfg.get("N_cells_x", 80)), int(cfg.get("N_cells_y", 80))
        shape = (nx + 5, ny + 5)
        r = oracle.Reference(text, shape)
        n, conv, log = r.run(iters)
        np.savez_compressed(HERE / f"run_{tag}.npz", u=r.get(0), v=r.get(1), p=r.get(2), log=log,
                            converged=np.array(conv), config=json.dumps(cfg))
        print(f"run_{tag}.npz", n, conv)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference"), sys.argv[2:])
