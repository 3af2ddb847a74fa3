"""The reference-side binding, run: simple-hpc's own run_simple against run_simple_sgpu.

simple-hpc_b200/adapter/sgpu_backend.cpp is what a simple-hpc maintainer adds to call this library
from the reference's main in place of run_simple_hip. oracle/Makefile (target `adapter`) compiles it
with the reference's own headers and sources, read in place, and links libsgpu.so into
oracle/_ref/adapter_check, which runs one config through the reference's CPU run_simple and through
the binding, then compares iterations, the converged flag, the residual log and u, v, p bit for bit.
The binding uses sampled timers (sgpu_set_profiling mode 2): the first 10 iterations are
host-issued and timed per phase, the rest replay the captured graph, so a run past 10 iterations
also checks that the switch carries the stopping rule's state (the iteration count and the
running_max maxima) over exactly.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from conftest import REPO, config_text, cuda_available, snapshot_config

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

CHECK = REPO / "oracle" / "_ref" / "adapter_check"


@pytest.mark.parametrize("case", ["runmax_mg", "absolute_rb_short", "cg"])
def test_binding_equals_reference_run_simple(tmp_path, case):
    if not CHECK.exists():
        pytest.skip("adapter_check was not built (no reference tree at build time)")
    cfg = snapshot_config("converged_32x40")  # running_max, tolerance 1e-4, Re 400, 32 x 40
    if case == "runmax_mg":
        cfg.update(momentum_solver="gs_multicolour", pressure_solver="mg")
    elif case == "absolute_rb_short":
        cfg.update(momentum_solver="gs_multicolour", pressure_solver="gs_redblack",
                   residual_normalisation="absolute", maxit="8")
    else:
        cfg.update(momentum_solver="gs_multicolour", pressure_solver="cg", maxit="40")
    cfg["backend"] = "gpu"
    cfg["output_dir"] = str(tmp_path / "out")
    path = Path(tmp_path) / "case.cfg"
    path.write_text(config_text(cfg))
    r = subprocess.run([str(CHECK), str(path)], capture_output=True, text=True, timeout=600)
    tail = "\n".join(r.stdout.splitlines()[-3:])
    print(tail)
    assert r.returncode == 0 and "adapter ok" in r.stdout, tail + r.stderr
