"""Config parsing and parameters: same keys, defaults, derived values and errors as the reference.

Mirrors simple-hpc tests/unit/test_config.cpp and test_params.cpp; where the reference build is
present (oracle/_ref), every case is also checked against the reference's own make_params.
"""
from __future__ import annotations

import ctypes as C

import pytest


def ref_params(oracle_mod, text: str):
    ints = (C.c_int * 26)()
    dbls = (C.c_double * 10)()
    L = oracle_mod.ref_lib()
    rc = L.ref_make_params(text.encode(), ints, dbls)
    if rc != 0:
        return None, L.ref_last_error().decode()
    return (list(ints), list(dbls)), None


def our_view(p):
    ints = [p.NX, p.NY, p.H, p.N_halo_x, p.N_halo_y, p.maxit_inner_u, p.maxit_inner_v,
            p.maxit_inner_p, p.maxit, p.convection_scheme, p.diffusion_order, p.hybrid_switch,
            p.residual_normalisation, p.backend, p.momentum_solver, p.pressure_solver,
            p.pressure_maxit, p.mg_cycles, p.mg_pre, p.mg_post, p.halo_overlap, p.write_fields,
            p.grid_rows_cfg, p.grid_cols_cfg, p.nrows, p.ncols]
    dbls = [p.Re, p.error_tolerance, p.relaxation_factor_u, p.relaxation_factor_v,
            p.relaxation_factor_p, p.pressure_tolerance, p.mg_omega, p.dx, p.dy, p.nu]
    return ints, dbls


CASES_OK = [
    "",
    "N_cells_x = 32\nN_cells_y = 40\nRe = 400\n",
    "  N_cells_x=7   # comment\n\n# only a comment\nN_cells_y =9\nconvection_scheme = UDS\n",
    "backend = gpu\nmomentum_solver = gs_multicolour\npressure_solver = mg\nmg_omega = 2\n",
    "residual_normalisation = running_max\nHybrid_switch = False\nmpi_grid = 2x3\n",
    "pressure_solver = cg\npressure_tolerance = 1e-9\npressure_maxit = 5\nwrite_fields = False\n",
    "error_tolerance = 0\nmaxit = 3\nrelaxation_factor_u = 0.7\nmpi_grid = auto\n",
    "diffusion_order = 2\nN_halo_x = 3\nN_halo_y = 3\nmg_pre = 0\nmg_post = 0\noutput_dir = a/b c\n",
]

CASES_ERR = [
    ("N_cells_x = 3\nN_cells_x = 4\n", "config line 2: duplicate key 'N_cells_x'"),
    ("N_cells_x 3\n", "config line 1: malformed line (expected key = value)"),
    ("N_cells_x = \n", "config line 1: malformed line (empty key or value)"),
    ("= 3\n", "config line 1: malformed line (empty key or value)"),
    ("foo = 1\n", "unknown config key: foo"),
    ("zeta = 1\nalpha = 2\n", "unknown config key: alpha"),
    ("N_cells_x = 3.5\n", "cannot parse integer for 'N_cells_x': 3.5"),
    ("Re = fast\n", "cannot parse number for 'Re': fast"),
    ("Hybrid_switch = yes\n", "invalid boolean for 'Hybrid_switch' (use True/False): yes"),
    ("convection_scheme = CDS\n", "unknown value for 'convection_scheme': CDS"),
    ("pressure_solver = sor\n", "unknown value for 'pressure_solver': sor"),
    ("N_halo_x = 3\n", "N_halo_x must equal N_halo_y"),
    ("N_halo_x = 1\nN_halo_y = 1\n", "halo width H must be >= 2"),
    ("diffusion_order = 3\n", "diffusion_order must be 2 or 4"),
    ("N_cells_x = 0\n", "N_cells_x and N_cells_y must be positive"),
    ("Hybrid_switch = True\n", "Hybrid_switch = True is not supported"),
    ("pressure_tolerance = 0\n", "pressure_tolerance must be positive"),
    ("pressure_maxit = 0\n", "pressure_maxit must be >= 1"),
    ("mg_cycles = 0\n", "mg_cycles must be >= 1"),
    ("mg_pre = -1\n", "mg_pre and mg_post must be >= 0"),
    ("mg_omega = 2.5\n", "mg_omega must be in (0, 2]"),
    ("mpi_grid = 2by2\n", "mpi_grid must be auto or RxC (e.g. 2x2): 2by2"),
    ("mpi_grid = 0x2\n", "mpi_grid sizes must be positive: 0x2"),
]


@pytest.mark.parametrize("text", CASES_OK)
def test_params_match_reference(sgpu_mod, oracle_mod, text):
    p = sgpu_mod.params_from_config(text)
    if oracle_mod.ref_available():
        ref, err = ref_params(oracle_mod, text)
        assert err is None, err
        assert our_view(p) == ref
    else:
        assert p.nrows == p.NX + 2 * p.H + 1 and p.dx == 1.0 / p.NY


@pytest.mark.parametrize("text,msg", CASES_ERR)
def test_param_errors_match_reference(sgpu_mod, oracle_mod, text, msg):
    with pytest.raises(sgpu_mod.SgpuError) as e:
        sgpu_mod.params_from_config(text)
    assert str(e.value) == msg
    if oracle_mod.ref_available():
        _, err = ref_params(oracle_mod, text)
        assert err == msg


def test_defaults(sgpu_mod):
    p = sgpu_mod.params_from_config("")
    assert (p.NX, p.NY, p.H, p.maxit, p.maxit_inner_p) == (80, 80, 2, 15000, 8)
    assert p.Re == 1000.0 and p.error_tolerance == 1e-4 and p.mg_omega == 1.8
    assert (p.nrows, p.ncols) == (85, 85) and p.nu == 1.0 / 1000.0
    assert p.precision == sgpu_mod.PREC_FP64 and p.mg_mode == 0 and p.warm_start == 0


def test_non_square_spacing(sgpu_mod):
    """dx = 1 / NY (column spacing), dy = 1 / NX (row spacing): test_boundary.cpp:17-24."""
    p = sgpu_mod.params_from_config("N_cells_x = 32\nN_cells_y = 48\n")
    assert p.dx == 1.0 / 48 and p.dy == 1.0 / 32 and (p.nrows, p.ncols) == (37, 53)


def test_build_only_keys(sgpu_mod):
    p = sgpu_mod.params_from_config("precision = mixed\nmg_mode = tolerance\nwarm_start = cnn\n"
                                    "cnn_weights = w.bin\ngraph_batch = 8\n")
    assert p.precision == sgpu_mod.PREC_MIXED and p.mg_mode == 1 and p.warm_start == 1
    assert p.cnn_weights == b"w.bin" and p.graph_batch == 8
    with pytest.raises(sgpu_mod.SgpuError, match="unknown value for 'precision'"):
        sgpu_mod.params_from_config("precision = fp16\n")
