"""Batched cavities (sgpu_batch_*): many independent cavities in one graph launch.

The batch applies the reference's stopping rule (run_outer_loop, solver.cpp:117-129) per cavity on
the device, so each cavity must end exactly where its own sgpu_run ends: in FP64 the iteration
count, the converged flag, every logged residual and the final u, v, p are bit-identical to the
single runs (which the parity suite ties to the reference). A mixed-precision batch is compared with
the single FP64 runs by its max and L2 relative error. The autotuner changes no bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bit_equal, config_text, cuda_available, snapshot_config

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def cavity(n: int, re: float, **kw) -> dict:
    cfg = snapshot_config("short_16")
    cfg.update(N_cells_x=str(n), N_cells_y=str(n), Re=str(re), convection_scheme="QUICK",
               diffusion_order="2", momentum_solver="gs_multicolour", pressure_solver="mg",
               error_tolerance="1e-5", maxit="4000")
    cfg.update({k: str(v) for k, v in kw.items()})
    return cfg


def single_run(sgpu_mod, cfg, maxit):
    p = sgpu_mod.params_from_config(config_text(cfg))
    with sgpu_mod.Solver(p) as s:
        res, log = s.run(maxit)
        return res, log, [s.download(f) for f in (0, 1, 2)]


CASES = [
    cavity(16, 100),
    cavity(24, 400),
    cavity(32, 100),
    cavity(20, 250, convection_scheme="UDS"),  # 2-colour sweeps
    cavity(16, 100, momentum_solver="jacobi", pressure_solver="jacobi"),
    cavity(24, 200, pressure_solver="gs_redblack", residual_normalisation="running_max", error_tolerance="1e-3"),
    cavity(18, 150, N_cells_y="30"),  # rectangular
]


def test_fp64_batch_bit_identical_to_single_runs(sgpu_mod):
    maxit = 4000
    params = [sgpu_mod.params_from_config(config_text(c)) for c in CASES]
    with sgpu_mod.Batch(params) as b:
        secs = b.run(maxit, log_cap=maxit)
        r = b.results()
        logs = b.log()
        fields = [[b.download(i, f) for f in (0, 1, 2)] for i in range(len(CASES))]
    print(f"{len(CASES)} cavities in {secs * 1e3:.1f} ms; iterations {r['iterations'].tolist()}")
    for i, cfg in enumerate(CASES):
        res, log, ref = single_run(sgpu_mod, cfg, maxit)
        assert r["iterations"][i] == res.iterations, f"cavity {i}"
        assert r["converged"][i] == bool(res.converged), f"cavity {i}"
        assert np.array_equal(r["residuals"][i], log[-1, 1:]), f"cavity {i}"
        assert np.array_equal(logs[i, :res.iterations], log), f"cavity {i}: residual log"
        assert not logs[i, res.iterations:].any()
        for a, e in zip(fields[i], ref):
            assert bit_equal(a, e), f"cavity {i}"


def test_maxit_caps_each_cavity(sgpu_mod):
    params = [sgpu_mod.params_from_config(config_text(c)) for c in CASES[:3]]
    with sgpu_mod.Batch(params) as b:
        b.run(7)
        r = b.results()
        u = b.download(1, 0)
    assert r["iterations"].tolist() == [7, 7, 7] and not r["converged"].any()
    _, _, ref = single_run(sgpu_mod, CASES[1], 7)
    assert bit_equal(u, ref[0])
    with sgpu_mod.Batch(params[:1]) as b:
        b.run(0)
        assert b.results()["iterations"].tolist() == [0]


def test_autotune_changes_no_bit(sgpu_mod):
    cases = [cavity(64, 300), cavity(96, 700), cavity(64, 300, precision="mixed")]
    params = [sgpu_mod.params_from_config(config_text(c)) for c in cases]
    out = []
    for tune in (False, True):
        with sgpu_mod.Batch(params) as b:
            if tune:
                chosen = b.autotune()
                print(f"autotuned row segments: {chosen}")
                assert all(s > 0 for s in chosen)
            b.run(40)
            out.append([[b.download(i, f) for f in (0, 1, 2)] for i in range(len(cases))])
    for a, e in zip(out[0], out[1]):
        for x, y in zip(a, e):
            assert bit_equal(x, y)


def test_mixed_batch_close_to_fp64_single_runs(sgpu_mod):
    cases = [cavity(32, 100), cavity(48, 400), cavity(64, 1000), cavity(40, 200, convection_scheme="UDS")]
    params = [sgpu_mod.params_from_config(config_text(dict(c, precision="mixed"))) for c in cases]
    with sgpu_mod.Batch(params) as b:
        b.autotune()
        secs = b.run(6000)
        r = b.results()
        fields = [[b.download(i, f) for f in (0, 1, 2)] for i in range(len(cases))]
    print(f"mixed batch: {secs * 1e3:.1f} ms, iterations {r['iterations'].tolist()}")
    for i, cfg in enumerate(cases):
        res, _, ref = single_run(sgpu_mod, cfg, 6000)
        assert res.converged and r["converged"][i]
        assert abs(int(r["iterations"][i]) - res.iterations) <= max(5, res.iterations // 50)
        for k, (a, e) in enumerate(zip(fields[i], ref)):
            mx = np.max(np.abs(a - e)) / np.max(np.abs(e))
            l2 = np.linalg.norm(a - e) / np.linalg.norm(e)
            print(f"cavity {i} field {k}: max rel {mx:.2e}, L2 rel {l2:.2e}")
            assert mx < 1e-6 and l2 < 1e-6


def test_batch_rejects_unsupported(sgpu_mod):
    for bad in (dict(pressure_solver="cg"), dict(mg_mode="tolerance")):
        p = sgpu_mod.params_from_config(config_text(cavity(16, 100, **bad)))
        with pytest.raises(sgpu_mod.SgpuError, match="batch"):
            sgpu_mod.Batch([p])


@pytest.mark.parametrize("extra", [{}, {"precision": "mixed"}, {"pressure_solver": "gs_redblack"}])
def test_run_graph_equals_host_loop(sgpu_mod, extra, capfd):
    """sgpu_run replays one captured outer iteration inside a WHILE graph with the stopping test on
    the device; with the per-phase timers on it issues every launch from the host. Both must give
    the same iterations, residual log and fields, bit for bit, also across print_every chunks."""
    cfg = cavity(32, 100, **extra)
    out = []
    for profiling in (True, False):
        p = sgpu_mod.params_from_config(config_text(cfg))
        with sgpu_mod.Solver(p) as s:
            s.set_profiling(profiling)
            res, log = s.run(4000, print_every=100)
            out.append((res.iterations, res.converged, log, [s.download(f) for f in (0, 1, 2)]))
    printed = capfd.readouterr().out.splitlines()
    (i0, c0, l0, f0), (i1, c1, l1, f1) = out
    assert i0 == i1 and c0 == c1 and c0
    assert np.array_equal(l0, l1)
    for a, b in zip(f0, f1):
        assert bit_equal(a, b)
    # the same progress lines from both paths
    half = len(printed) // 2
    assert printed[:half] == printed[half:] and printed[0].startswith("iter 1 ")
