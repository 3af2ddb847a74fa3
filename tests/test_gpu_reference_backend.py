"""The reference's own GPU backend, built for sm_100a, against this repository's FP64 solver.

simple-hpc's HipSolver (src/hip/solver_hip.hip, gs_multicolour + gs_redblack only) is compiled by
oracle/Makefile as CUDA with the flags of its own CUDA build (-DSIMPLE_CUDA --fmad=false) and timed
by bench.py as the reference GPU baseline on the same B200. Its per-cell arithmetic follows the CPU
code expression for expression, so its fields equal the CPU's bit for bit while its residual sums
use another order (the reference's own GPU test accepts 1e-12 relative on them,
tests/hip/test_hip.cpp:68). This repository's FP64 path reproduces the CPU bits, residuals included,
so after the same iterations both GPU solvers must hold identical fields, and the residuals must
agree to 1e-12.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bit_equal, config_text, cuda_available, describe_diff

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.mark.parametrize("n,iters", [(64, 10), (256, 5)])
def test_reference_gpu_backend_equals_ours(sgpu_mod, oracle_mod, n, iters):
    if not oracle_mod.refgpu_available():
        pytest.skip("the reference GPU backend was not built (no reference tree at build time)")
    cfg = {"N_cells_x": n, "N_cells_y": n, "Re": 1000, "convection_scheme": "QUICK", "diffusion_order": 4,
           "momentum_solver": "gs_multicolour", "pressure_solver": "gs_redblack", "error_tolerance": 0,
           "maxit": iters}
    text = config_text(cfg)
    p = sgpu_mod.params_from_config(text)
    ref = oracle_mod.ReferenceGpu(text, p.shape)
    _, rres = ref.iterations(iters)
    theirs = [ref.get(f) for f in (0, 1, 2)]
    ref.close()
    with sgpu_mod.Solver(p) as g:
        res, log = g.run(iters)
        ours = [g.download(f) for f in (0, 1, 2)]
    for name, a, b in zip("uvp", ours, theirs):
        assert bit_equal(a, b), f"{name}: " + describe_diff(a, b)
    rel = np.abs(log[:, 1:] - rres) / np.maximum(np.abs(rres), 1e-300)
    assert rel.max() <= 1e-12, rel.max()
