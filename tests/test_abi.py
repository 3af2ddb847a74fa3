"""The C-ABI library loads on any machine and exports every function include/sgpu.h declares.

No compute call runs here: without a GPU, creating a solver must fail cleanly with
SGPU_E_NODEVICE and a message (never a crash or a silent CPU path).
"""
from __future__ import annotations

import ctypes as C
import re

import pytest

from conftest import REPO, cuda_available


def declared_functions() -> list[str]:
    text = (REPO / "include" / "sgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sgpu_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["sgpu_create", "sgpu_destroy", "sgpu_assemble_u", "sgpu_bc_u", "sgpu_residual_u",
                 "sgpu_sweep_u", "sgpu_assemble_v", "sgpu_bc_v", "sgpu_residual_v", "sgpu_sweep_v",
                 "sgpu_assemble_p", "sgpu_solve_p", "sgpu_correct", "sgpu_outer_iteration",
                 "sgpu_run", "sgpu_download", "sgpu_params_from_config"]:
        assert must in names


def test_library_exports_every_declared_symbol(sgpu_mod):
    lib = C.CDLL(str(sgpu_mod.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared in include/sgpu.h but not exported: {missing}"


def test_version_and_errors(sgpu_mod):
    assert b"sm_100a" in sgpu_mod.lib().sgpu_version()
    with pytest.raises(sgpu_mod.SgpuError, match="unknown config key: nope"):
        sgpu_mod.params_from_config("nope = 1\n")
    assert sgpu_mod.lib().sgpu_last_error() == b"unknown config key: nope"


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU path")
def test_create_without_gpu_fails_cleanly(sgpu_mod):
    p = sgpu_mod.params_from_config("momentum_solver = gs_multicolour\npressure_solver = mg\n"
                                    "N_cells_x = 8\nN_cells_y = 8\n")
    with pytest.raises(sgpu_mod.SgpuError) as e:
        sgpu_mod.Solver(p)
    assert e.value.code in (sgpu_mod.E_NODEVICE, sgpu_mod.E_CUDA)


def test_mg_levels_without_gpu(sgpu_mod):
    assert sgpu_mod.mg_levels(32, 40) == [(32, 40), (16, 20), (8, 10), (4, 5)]
