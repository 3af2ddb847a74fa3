"""The oracle (C restatement) against the reference's own golden data — the parity pin.

* The reference's committed regression snapshots (short_16: 16x16, 10 iterations; converged_32x40:
  32 x 40, Re 400, 725 iterations to running_max 1e-4; both gs_lex / gs_lex) must be reproduced bit
  for bit, residual log included (simple-hpc tests/regression/test_snapshots.cpp pins the same).
* Runs of the reference's own sources for the GPU solver combinations (fixtures made by
  tests/golden/make_golden.py) must be reproduced bit for bit.
* Coefficient known answers from simple-hpc tests/unit/test_coefficients.cpp.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bit_equal, config_text, describe_diff, load_golden


def run_oracle(sgpu_mod, oracle_mod, cfg: dict, iters: int):
    p = sgpu_mod.params_from_config(config_text(cfg))
    o = oracle_mod.Oracle(p)
    n, conv, log = o.run(iters)
    return o, n, conv, log


@pytest.mark.parametrize("name", ["short_16", "converged_32x40"])
def test_snapshot_bit_exact(sgpu_mod, oracle_mod, name):
    g = load_golden(f"snapshot_{name}.npz")
    cfg = g["config"]
    o, n, conv, log = run_oracle(sgpu_mod, oracle_mod, cfg, int(cfg["maxit"]))
    assert n == g["alog"].shape[0]
    assert bit_equal(log, g["alog"]), describe_diff(log, g["alog"])
    for k, fid in (("u", 0), ("v", 1), ("p", 2)):
        assert bit_equal(o.get(fid), g[k]), f"{k}: " + describe_diff(o.get(fid), g[k])


@pytest.mark.parametrize("tag", ["mc_rb_quick4_32x40", "mc_mg_quick4_32x40", "mc_cg_uds2_32x40",
                                 "jac_jac_quick4_16", "cavity32_re100_mc_mg", "runmax_mc_mg_32x40",
                                 "runmax_mc_rb_32x40"])
def test_reference_runs_bit_exact(sgpu_mod, oracle_mod, tag):
    g = load_golden(f"run_{tag}.npz")
    cfg = g["config"]
    o, n, conv, log = run_oracle(sgpu_mod, oracle_mod, cfg, int(cfg["maxit"]))
    assert n == g["log"].shape[0]
    assert conv == bool(g["converged"])
    assert bit_equal(log, g["log"]), describe_diff(log, g["log"])
    for k, fid in (("u", 0), ("v", 1), ("p", 2)):
        assert bit_equal(o.get(fid), g[k]), f"{k}: " + describe_diff(o.get(fid), g[k])


def test_config1_converges_in_494_iterations():
    """32x32 Re 100 QUICK/2 gs_multicolour + mg to 1e-5: the reference needs 494 iterations."""
    g = load_golden("run_cavity32_re100_mc_mg.npz")
    assert g["log"].shape[0] == 494 and bool(g["converged"])


def _kat_params(sgpu_mod, scheme: int, order: int):
    # The hand-set Params of test_coefficients.cpp:10-23 (NX = NY = 8, dx 0.125, dy 0.25, nu 0.01).
    p = sgpu_mod.Params()
    sgpu_mod.lib().sgpu_params_default(p)
    p.NX = p.NY = 8
    p.H = p.N_halo_x = p.N_halo_y = 2
    p.dx, p.dy, p.nu = 0.125, 0.25, 0.01
    p.convection_scheme, p.diffusion_order = scheme, order
    return p


def _conv(oracle_mod, p, ue, uw, vn, vs, i, j):
    import ctypes as C
    out = (C.c_double * 9)()
    oracle_mod.orc_lib().orc_convective(C.byref(p), ue, uw, vn, vs, i, j, out)
    return dict(zip(["AE", "AW", "AN", "AS", "AEE", "AWW", "ANN", "ASS", "AP"], list(out)))


def _diff(oracle_mod, p, i, j):
    import ctypes as C
    out = (C.c_double * 9)()
    oracle_mod.orc_lib().orc_diffusive(C.byref(p), i, j, out)
    return dict(zip(["AE", "AW", "AN", "AS", "AEE", "AWW", "ANN", "ASS", "AP"], list(out)))


def test_coefficient_known_answers(sgpu_mod, oracle_mod):
    import ctypes as C
    L = oracle_mod.orc_lib()
    p = _kat_params(sgpu_mod, sgpu_mod.QUICK, 4)
    band = lambda i, j: L.orc_in_boundary_band(C.byref(p), i, j)  # noqa: E731
    assert band(2, 5) and band(9, 5) and band(5, 3) and band(5, 10)
    assert not band(5, 2) and not band(5, 5)

    p = _kat_params(sgpu_mod, sgpu_mod.UDS, 2)
    c = _conv(oracle_mod, p, 1.0, 2.0, 3.0, 4.0, 5, 5)
    assert c["AE"] == 0.0 and c["AN"] == 0.0
    assert c["AW"] == pytest.approx(0.25 * 2.0) and c["AS"] == pytest.approx(0.125 * 4.0)
    assert c["AP"] == pytest.approx(1.0)
    c = _conv(oracle_mod, p, -1.0, -2.0, -3.0, -4.0, 5, 5)
    assert c["AE"] == pytest.approx(0.25) and c["AW"] == 0.0
    assert c["AN"] == pytest.approx(0.375) and c["AS"] == 0.0 and c["AP"] == pytest.approx(0.625)

    p = _kat_params(sgpu_mod, sgpu_mod.QUICK, 4)
    c = _conv(oracle_mod, p, 1.0, 1.0, 1.0, 1.0, 5, 5)
    assert c["AE"] == pytest.approx(-0.25 * 0.375)
    assert c["AW"] == pytest.approx(-0.25 * (-0.125 - 0.75))
    assert c["AN"] == pytest.approx(-0.125 * 0.375)
    assert c["AS"] == pytest.approx(-0.125 * (-0.125 - 0.75))
    assert c["AEE"] == 0.0 and c["AWW"] == pytest.approx(-0.125 * 0.25)
    assert c["ASS"] == pytest.approx(-0.125 * 0.125)
    assert c["AP"] == pytest.approx(c["AE"] + c["AW"] + c["AN"] + c["AS"] + c["AWW"] + c["ASS"])
    c = _conv(oracle_mod, p, -1.0, 2.0, -3.0, 4.0, 2, 5)  # band: UDS fallback
    assert c["AE"] == pytest.approx(0.25) and c["AW"] == pytest.approx(0.5) and c["AEE"] == 0.0
    assert c["AP"] == pytest.approx(0.25 + 0.5 + 0.375 + 0.5)

    p = _kat_params(sgpu_mod, sgpu_mod.UDS, 2)
    d = _diff(oracle_mod, p, 5, 5)
    assert d["AE"] == pytest.approx(0.25 * 0.01 / 0.125)
    assert d["AN"] == pytest.approx(0.125 * 0.01 / 0.25)
    assert d["AP"] == pytest.approx(0.01 * (2 * 0.125 / 0.25 + 2 * 0.25 / 0.125))
    p.diffusion_order = 4
    d = _diff(oracle_mod, p, 5, 5)
    assert d["AE"] == pytest.approx(4.0 / 3 * 0.25 * 0.01 / 0.125)
    assert d["AEE"] == pytest.approx(-1.0 / 12 * 0.25 * 0.01 / 0.125)
    assert d["ANN"] == pytest.approx(-1.0 / 12 * 0.125 * 0.01 / 0.25)
    assert d["AP"] == pytest.approx(0.01 * (2.5 * 0.125 / 0.25 + 2.5 * 0.25 / 0.125))
    assert _diff(oracle_mod, p, 5, 3)["AEE"] == 0.0
    assert _diff(oracle_mod, p, 5, 2)["AEE"] != 0.0


def test_colourings_separate_stencil_offsets():
    """Every stencil neighbour of a cell has another colour (test_inner_solvers.cpp:60-76)."""
    offsets5 = [(0, 1), (0, -1), (0, 2), (0, -2), (1, 0), (-1, 0), (2, 0), (-2, 0)]
    for i in range(10):
        for j in range(10):
            c = (i + 3 * j) % 5
            for di, dj in offsets5:
                assert (i + di + 3 * (j + dj)) % 5 != c
            c2 = (i + j) % 2
            for di, dj in offsets5[:2] + offsets5[4:6]:
                assert (i + di + j + dj) % 2 != c2


def test_mg_level_dims(sgpu_mod, oracle_mod):
    """mg_level_dims (multigrid.cpp:143-151), as pinned by test_multigrid.cpp:75-88."""
    import ctypes as C
    dims = (C.c_int * 128)()

    def orc(nx, ny):
        n = oracle_mod.orc_lib().orc_mg_level_dims(nx, ny, dims)
        return [(dims[2 * k], dims[2 * k + 1]) for k in range(n)]

    assert orc(64, 64) == [(64, 64), (32, 32), (16, 16), (8, 8), (4, 4)]
    assert orc(32, 40) == [(32, 40), (16, 20), (8, 10), (4, 5)]
    assert orc(9, 11) == [(9, 11)]
    assert orc(4096, 4096)[-1] == (4, 4) and len(orc(4096, 4096)) == 11
    assert len(orc(1024, 1024)) == 9
    for nx, ny in [(64, 64), (32, 40), (9, 11), (4096, 4096), (48, 80), (6, 6), (8, 4)]:
        assert sgpu_mod.mg_levels(nx, ny) == orc(nx, ny)


def test_ordered_sum_is_row_then_rows(oracle_mod):
    rng = np.random.default_rng(7)
    v = rng.standard_normal((37, 53)) * 10.0 ** rng.integers(-8, 8, (37, 53))
    expect = 0.0
    for r in range(v.shape[0]):
        s = 0.0
        for c in range(v.shape[1]):
            s += v[r, c]
        expect += s
    assert oracle_mod.ordered_sum(v) == expect
