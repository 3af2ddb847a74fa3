"""Divergence detection: a run whose residuals become NaN or Inf stops with SGPU_E_NONFINITE.

The reference has no such test: a diverged case runs on to maxit with NaN residuals (simple-hpc
docs/RESULTS.md:237-245 reports 32^2 at relaxation 0.7 / 0.2 diverging to NaN within 400 iterations).
Here sgpu_run stops after the first iteration whose residuals are not all finite, with the result and
the log covering the iterations run, in both run paths: the graph replay (stopping test on the
device) and the host-issued loop (profiling on). The batch engine marks such a cavity diverged and
lets the others finish. Failures are made on the host or by the physics, never by a GPU fault: the
genuine divergence of the documented case, and a NaN uploaded into u between runs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import bit_equal, config_text, cuda_available, describe_diff

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DIVERGING = {"N_cells_x": 32, "N_cells_y": 32, "Re": 1000, "convection_scheme": "QUICK",
             "diffusion_order": 4, "momentum_solver": "gs_multicolour", "pressure_solver": "mg",
             "relaxation_factor_u": 0.7, "relaxation_factor_v": 0.7, "relaxation_factor_p": 0.2,
             "error_tolerance": 1e-5, "maxit": 1000}


def raw_run(sgpu_mod, solver, maxit):
    """sgpu_run through the C ABI, keeping the result and the log when the call fails."""
    log = np.zeros((maxit, 4))
    res = sgpu_mod.Result()
    rc = sgpu_mod.lib().sgpu_run(solver._h, maxit, log.ctypes.data_as(C.POINTER(C.c_double)), 0,
                                 C.byref(res))
    return rc, res, log[:res.iterations].copy()


@pytest.fixture(scope="module")
def oracle_divergence(oracle_mod, sgpu_mod):
    p = sgpu_mod.params_from_config(config_text(DIVERGING))
    o = oracle_mod.Oracle(p)
    n, conv, log = o.run(1000)
    finite = np.isfinite(log[:, 1:]).all(axis=1)
    first_bad = int(np.argmin(finite)) + 1  # 1-based iteration of the first non-finite residual
    assert not finite.all() and first_bad < 400
    return first_bad, log


@pytest.mark.parametrize("profiled", [False, True])
def test_diverged_run_stops_where_the_oracle_first_goes_nonfinite(sgpu_mod, oracle_divergence, profiled):
    first_bad, olog = oracle_divergence
    p = sgpu_mod.params_from_config(config_text(DIVERGING))
    with sgpu_mod.Solver(p) as g:
        g.set_profiling(profiled)
        rc, res, log = raw_run(sgpu_mod, g, 1000)
        assert rc == sgpu_mod.E_NONFINITE, sgpu_mod.lib().sgpu_last_error().decode()
        msg = sgpu_mod.lib().sgpu_last_error().decode()
        assert f"outer iteration {first_bad}" in msg
        assert res.iterations == first_bad and not res.converged
        # the finite part of the log is the oracle's, bit for bit
        assert bit_equal(log[:first_bad - 1], olog[:first_bad - 1]), describe_diff(log[:first_bad - 1],
                                                                                  olog[:first_bad - 1])
        assert not np.isfinite(log[first_bad - 1, 1:]).all()
    # the context stays usable: a new solver on the same device runs normally
    with sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(dict(DIVERGING, Re=100)))) as g2:
        rc2, res2, _ = raw_run(sgpu_mod, g2, 10)
        assert rc2 == 0 and res2.iterations == 10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_uploaded_between_runs_stops_the_next_run(sgpu_mod, precision):
    cfg = dict(DIVERGING, Re=100, relaxation_factor_u=0.3, relaxation_factor_v=0.3, precision=precision)
    p = sgpu_mod.params_from_config(config_text(cfg))
    with sgpu_mod.Solver(p) as g:
        res, _ = g.run(5)
        assert res.iterations == 5
        u = g.download(sgpu_mod.F_U)
        u[p.H + 7, p.H + 9] = np.nan
        g.upload(sgpu_mod.F_U, u)
        rc, res, log = raw_run(sgpu_mod, g, 50)
        assert rc == sgpu_mod.E_NONFINITE
        assert res.iterations == 1 and log.shape[0] == 1 and not np.isfinite(log[0, 1:]).all()
        with pytest.raises(sgpu_mod.SgpuError, match="NaN or Inf"):
            g.run(50)


def test_batch_marks_the_diverged_cavity_and_finishes_the_others(sgpu_mod, oracle_divergence):
    first_bad, _ = oracle_divergence
    good = dict(DIVERGING, Re=100, relaxation_factor_u=0.3, relaxation_factor_v=0.3)
    cfgs = [good, DIVERGING, dict(good, N_cells_x=24)]
    params = [sgpu_mod.params_from_config(config_text(c)) for c in cfgs]
    with sgpu_mod.Batch(params) as b:
        b.run(1000)
        r = b.results()
        assert r["diverged"].tolist() == [False, True, False]
        assert r["iterations"][1] == first_bad and not r["converged"][1]
        for i in (0, 2):
            with sgpu_mod.Solver(params[i]) as s:
                res, _ = s.run(1000)
                assert r["converged"][i] and res.converged and r["iterations"][i] == res.iterations
                assert bit_equal(b.download(i, sgpu_mod.F_U), s.download(sgpu_mod.F_U))
