"""Mixed precision (precision = mixed): FP32 inner solves inside FP64 defect correction.

The mixed path is not bit-identical to the reference by design; these tests bound its distance from
the FP64 oracle and check that it converges like the FP64 method:
* the 32 x 32, Re 100, QUICK / 2, gs_multicolour + mg case (494 FP64 iterations to 1e-5) converges
  in about as many iterations and to the FP64 fields within a small relative error;
* fixed work on the 32 x 40 snapshot case stays close to the FP64 trajectory;
* the residuals the stopping test reads are computed in FP64: the first iteration's res_u and res_v,
  which do not depend on any inner solve, equal the oracle's to FP64 rounding (the mixed path adds
  the per-cell |R| in a fixed tree instead of the reference's row-by-row chain).
Errors are reported as max |a - b| / max |b| (relative to the field's scale) and L2 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bit_equal, config_text, cuda_available, load_golden, snapshot_config

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def rel_errors(a: np.ndarray, b: np.ndarray) -> tuple[float, float]:
    scale = np.max(np.abs(b))
    mx = float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a - b)))
    l2 = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return mx, l2


def test_mixed_converges_like_fp64(sgpu_mod):
    g = load_golden("run_cavity32_re100_mc_mg.npz")
    cfg = dict(g["config"])
    cfg["precision"] = "mixed"
    p = sgpu_mod.params_from_config(config_text(cfg))
    with sgpu_mod.Solver(p) as s:
        res, log = s.run(p.maxit)
        fields = {k: s.download(f) for k, f in (("u", 0), ("v", 1), ("p", 2))}
    n64 = g["log"].shape[0]
    print(f"mixed: {res.iterations} iterations (FP64: {n64})")
    assert res.converged
    assert abs(res.iterations - n64) <= max(5, n64 // 50)
    for k in ("u", "v", "p"):
        mx, l2 = rel_errors(fields[k], g[k])
        print(f"{k}: max rel {mx:.3e}, L2 rel {l2:.3e}")
        assert mx < 1e-6 and l2 < 1e-6


def test_mixed_fixed_work_close_to_fp64(sgpu_mod, oracle_mod):
    cfg = snapshot_config("converged_32x40")
    cfg.update(momentum_solver="gs_multicolour", pressure_solver="mg", error_tolerance="0",
               maxit="60")
    p64 = sgpu_mod.params_from_config(config_text(cfg))
    o = oracle_mod.Oracle(p64)
    _, _, olog = o.run(60)
    cfg["precision"] = "mixed"
    p = sgpu_mod.params_from_config(config_text(cfg))
    with sgpu_mod.Solver(p) as s:
        res, log = s.run(60)
        fields = {k: s.download(f) for k, f in (("u", 0), ("v", 1), ("p", 2))}
    # The first iteration's momentum residuals are computed before any inner solve: FP64 values,
    # summed in a different order than the oracle's chain (each of 1280 terms rounds once).
    diff = np.abs(log[0, 1:3] - olog[0, 1:3])
    print(f"first-iteration res_u, res_v: {log[0, 1:3]} vs {olog[0, 1:3]}")
    assert np.all(diff <= 1e-13 * np.abs(olog[0, 1:3]))
    for k, f in (("u", 0), ("v", 1), ("p", 2)):
        mx, l2 = rel_errors(fields[k], o.get(f))
        print(f"{k}: max rel {mx:.3e}, L2 rel {l2:.3e}")
        assert mx < 1e-6 and l2 < 1e-6
    rel = np.abs(log[:, 1:] - olog[:, 1:]) / np.maximum(np.abs(olog[:, 1:]), 1e-300)
    print(f"residual log max rel {rel.max():.3e}")
    assert rel.max() < 1e-4


@pytest.mark.parametrize("nx,ny,scheme,order", [(96, 160, "QUICK", 4), (130, 600, "UDS", 2)])
def test_mixed_large_grids_close_to_fp64(sgpu_mod, nx, ny, scheme, order):
    """Fixed work (20 iterations of the transient): the mixed trajectory against the FP64 one. The
    two inner solvers differ (FP32 sweeps and V-cycles), so mid-transient fields differ by a few
    1e-7 and the bound here is 2e-6; converged fields are held to 1e-6 (test_mixed_converges_like_fp64,
    the Ghia runs of tests/test_ghia.py)."""
    base = snapshot_config("short_16")
    base.update(N_cells_x=str(nx), N_cells_y=str(ny), Re="1000", convection_scheme=scheme,
                diffusion_order=str(order), momentum_solver="gs_multicolour", pressure_solver="mg",
                maxit="20", error_tolerance="0")
    p64 = sgpu_mod.params_from_config(config_text(base))
    with sgpu_mod.Solver(p64) as s:
        s.run(20)
        ref = {f: s.download(f) for f in (0, 1, 2)}
    base["precision"] = "mixed"
    p = sgpu_mod.params_from_config(config_text(base))
    with sgpu_mod.Solver(p) as s:
        s.run(20)
        for f in (0, 1, 2):
            mx, l2 = rel_errors(s.download(f), ref[f])
            print(f"field {f}: max rel {mx:.3e}, L2 rel {l2:.3e}")
            assert mx < 2e-6 and l2 < 2e-6


def test_mixed_rejects_other_solvers(sgpu_mod):
    cfg = snapshot_config("short_16")
    cfg.update(momentum_solver="gs_multicolour", pressure_solver="gs_redblack", precision="mixed")
    with pytest.raises(sgpu_mod.SgpuError, match="precision = mixed needs"):
        sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(cfg)))


@pytest.mark.parametrize("scheme,order", [("QUICK", 4), ("UDS", 2)])
def test_mixed_runs_repeat_bit_for_bit(sgpu_mod, scheme, order):
    """The mixed mode's sums are fixed FP64 trees and its sweeps a fixed schedule: two runs of the
    same case give the same residual log and fields bit for bit (on a grid with several strips and
    segments per sweep)."""
    base = snapshot_config("short_16")
    base.update(N_cells_x="300", N_cells_y="520", Re="1000", convection_scheme=scheme,
                diffusion_order=str(order), momentum_solver="gs_multicolour", pressure_solver="mg",
                precision="mixed", maxit="12", error_tolerance="0")
    out = []
    for _ in range(2):
        with sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(base))) as s:
            _, log = s.run(12)
            out.append((log, [s.download(f) for f in (0, 1, 2)]))
    (l0, f0), (l1, f1) = out
    assert bit_equal(l0, l1)
    for a, b in zip(f0, f1):
        assert bit_equal(a, b)


@pytest.mark.parametrize("nx,ny,scheme,order", [(77, 131, "QUICK", 4), (64, 95, "UDS", 2), (33, 2, "QUICK", 2)])
def test_mixed_odd_grids_close_to_fp64(sgpu_mod, nx, ny, scheme, order):
    """Grids whose column counts give the column-pair kernels (assemble_p, correct: two adjacent
    cells per thread, 16-byte FP64 accesses) a last pair with one cell as well as two, and a grid two
    cells wide: 10 iterations of the transient against the FP64 run."""
    base = snapshot_config("short_16")
    base.update(N_cells_x=str(nx), N_cells_y=str(ny), Re="400", convection_scheme=scheme,
                diffusion_order=str(order), momentum_solver="gs_multicolour", pressure_solver="mg",
                maxit="10", error_tolerance="0")
    p64 = sgpu_mod.params_from_config(config_text(base))
    with sgpu_mod.Solver(p64) as s:
        s.run(10)
        ref = {f: s.download(f) for f in (0, 1, 2)}
    base["precision"] = "mixed"
    p = sgpu_mod.params_from_config(config_text(base))
    with sgpu_mod.Solver(p) as s:
        s.run(10)
        for f in (0, 1, 2):
            mx, l2 = rel_errors(s.download(f), ref[f])
            print(f"field {f}: max rel {mx:.3e}, L2 rel {l2:.3e}")
            assert mx < 2e-6 and l2 < 2e-6


@pytest.mark.parametrize("nx,ny,pre,post", [(128, 128, 2, 2), (96, 160, 2, 2), (520, 96, 2, 2), (512, 512, 2, 2),
                                            (128, 128, 1, 3), (256, 256, 3, 0)])
def test_cluster_tail_matches_single_cta_tail(sgpu_mod, monkeypatch, nx, ny, pre, post):
    """The float V-cycle's levels of at most 65536 cells on one 16-CTA cluster (bands of rows with
    ghost rows in distributed shared memory; the levels of at most 1024 cells and the coarsest solve
    on one CTA) against the streamed levels and the single-CTA tail (SGPU_MG_CLUSTER=0): the same
    passes in the same colour order with the same per-cell expressions, which give the same bits
    (residual log and fields) after 8 outer iterations."""
    base = snapshot_config("short_16")
    base.update(N_cells_x=str(nx), N_cells_y=str(ny), Re="1000", convection_scheme="QUICK",
                diffusion_order="4", momentum_solver="gs_multicolour", pressure_solver="mg",
                maxit="8", error_tolerance="0", precision="mixed", mg_pre=str(pre), mg_post=str(post))
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("SGPU_MG_CLUSTER", flag)
        with sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(base))) as s:
            _, log = s.run(8)
            out[flag] = (log, [s.download(f) for f in (0, 1, 2)])
    (l0, f0), (l1, f1) = out["0"], out["1"]
    assert bit_equal(l0, l1)
    for a, b in zip(f0, f1):
        mx, l2 = rel_errors(b, a)
        print(f"cluster vs single-CTA tail: max rel {mx:.3e}, L2 rel {l2:.3e}")
        assert bit_equal(a, b)


@pytest.mark.parametrize("nx,ny,scheme,order,inner", [(128, 128, "QUICK", 4, 4), (96, 160, "QUICK", 2, 3),
                                                      (520, 96, "UDS", 2, 4), (33, 7, "QUICK", 4, 2),
                                                      (256, 256, "QUICK", 4, 4), (128, 128, "QUICK", 4, 1),
                                                      (64, 64, "UDS", 2, 5)])
def test_cluster_sweep_matches_streaming_sweep(sgpu_mod, monkeypatch, nx, ny, scheme, order, inner):
    """A small grid's correction sweeps on one 16-CTA cluster (bands of rows with two ghost rows in
    distributed shared memory, colour by colour, one launch per component) against the streaming
    sweep kernel (SGPU_CORR_CLUSTER=0): the same colour order and per-cell expression, so the same
    residual log and fields after 8 outer iterations, for five and two colours and a grid whose bands
    are two rows high."""
    base = snapshot_config("short_16")
    base.update(N_cells_x=str(nx), N_cells_y=str(ny), Re="1000", convection_scheme=scheme,
                diffusion_order=str(order), momentum_solver="gs_multicolour", pressure_solver="mg",
                maxit="8", error_tolerance="0", precision="mixed", maxit_inner_u=str(inner),
                maxit_inner_v=str(inner))
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("SGPU_CORR_CLUSTER", flag)
        with sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(base))) as s:
            _, log = s.run(8)
            out[flag] = (log, [s.download(f) for f in (0, 1, 2)])
    (l0, f0), (l1, f1) = out["0"], out["1"]
    for a, b in zip(f0, f1):
        mx, l2 = rel_errors(b, a)
        print(f"cluster vs streaming sweep: max rel {mx:.3e}, L2 rel {l2:.3e}")
    assert bit_equal(l0, l1)
    for a, b in zip(f0, f1):
        assert bit_equal(a, b)
