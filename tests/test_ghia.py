"""Ghia et al. (1982) validation of the lid-driven cavity at 80 x 80 (simple-hpc's `ghia_*` tests).

The reference validates its converged centrelines against the published Ghia data with its own
postprocess/validate_ghia.py, at Re 400 and 1000 on 80 x 80 cells, with rms limits 0.010 / 0.010
(Re 400) and 0.025 / 0.015 (Re 1000) for u and v (CMakeLists.txt:124-150). The configuration is
configs/validation/re{400,1000}_80.cfg with the solver keys overridden per test.

The check is split in two, because the reference tree (and so validate_ghia.py and its data) exists
only where the repository is built, not on the GPU machine:
* ``-m gpu``: the B200 solver run to convergence at 80 x 80 reproduces the oracle's run bit for
  bit: the same stopping iteration, residual log and u, v, p. The mixed-precision solve converges
  to the same fields within 1e-6 relative.
* CPU, where the reference tree is present: the oracle's converged run, written by this
  repository's output writer (byte-identical to the reference's writer), passes the reference's
  validate_ghia.py, run in place with --check and the reference's limits.
Together they validate the GPU path against Ghia's data without a copy of that data.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import bit_equal, config_text, cuda_available, describe_diff

REF_DIR = Path(os.environ.get("SIMPLE_HPC_REF", "/root/reference"))

# (Re, momentum_solver, pressure_solver, max rms u, max rms v): the multicolour and multigrid
# variants of the reference's ghia tests (CMakeLists.txt:141-150).
CASES = [(400, "gs_multicolour", "gs_redblack", 0.010, 0.010),
         (1000, "gs_multicolour", "gs_redblack", 0.025, 0.015),
         (400, "gs_multicolour", "mg", 0.010, 0.010),
         (1000, "gs_multicolour", "mg", 0.025, 0.015)]


def validation_config(re: int, ms: str, ps: str) -> dict:
    """configs/validation/re{re}_80.cfg with the solver keys of the test."""
    return {"N_cells_x": 80, "N_cells_y": 80, "Re": re, "maxit": 60000, "convection_scheme": "QUICK",
            "diffusion_order": 4, "N_halo_x": 2, "N_halo_y": 2, "maxit_inner_u": 4,
            "maxit_inner_v": 4, "maxit_inner_p": 8, "error_tolerance": 1e-5,
            "relaxation_factor_u": 0.3, "relaxation_factor_v": 0.3, "relaxation_factor_p": 0.2,
            "Hybrid_switch": "False", "momentum_solver": ms, "pressure_solver": ps,
            "residual_normalisation": "absolute"}


def rel_errors(a: np.ndarray, b: np.ndarray) -> tuple[float, float]:
    return (float(np.max(np.abs(a - b)) / np.max(np.abs(b))),
            float(np.linalg.norm(a - b) / np.linalg.norm(b)))


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("re,ms,ps,max_u,max_v", CASES)
def test_gpu_ghia_runs_equal_the_oracle(sgpu_mod, oracle_mod, re, ms, ps, max_u, max_v):
    cfg = validation_config(re, ms, ps)
    p = sgpu_mod.params_from_config(config_text(cfg))
    o = oracle_mod.Oracle(p)
    n, conv, olog = o.run(p.maxit)
    assert conv
    with sgpu_mod.Solver(p) as g:
        res, glog = g.run(p.maxit)
        assert res.converged and res.iterations == n
        assert bit_equal(glog, olog), describe_diff(glog, olog)
        for f in (0, 1, 2):
            a = g.download(f)
            assert bit_equal(a, o.get(f)), f"field {f}: " + describe_diff(a, o.get(f))
    if ps == "mg":
        cfg["precision"] = "mixed"
        with sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(cfg))) as m:
            res, _ = m.run(p.maxit)
            assert res.converged and abs(res.iterations - n) <= max(5, n // 50)
            for f in (0, 1, 2):
                mx, l2 = rel_errors(m.download(f), o.get(f))
                assert mx < 1e-6 and l2 < 1e-6, (f, mx, l2)


@pytest.mark.skipif(not (REF_DIR / "postprocess" / "validate_ghia.py").exists(),
                    reason="the reference tree (validate_ghia.py and the Ghia data) is not present")
@pytest.mark.parametrize("re,ms,ps,max_u,max_v", CASES)
def test_oracle_ghia_run_passes_validate_ghia(sgpu_mod, oracle_mod, tmp_path, re, ms, ps, max_u, max_v):
    cfg = validation_config(re, ms, ps)
    p = sgpu_mod.params_from_config(config_text(cfg))
    o = oracle_mod.Oracle(p)
    n, conv, log = o.run(p.maxit)
    assert conv
    out = tmp_path / f"re{re}_80_{ps}"
    p.output_dir = str(out).encode()
    res = sgpu_mod.Result()
    res.iterations, res.converged = n, 1
    sgpu_mod.write_outputs(p, o.get(0), o.get(1), o.get(2), log, res)
    r = subprocess.run([sys.executable, str(REF_DIR / "postprocess" / "validate_ghia.py"), str(out),
                        "--check", "--max-rms-u", str(max_u), "--max-rms-v", str(max_v)],
                       capture_output=True, text=True, cwd=str(tmp_path))
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
