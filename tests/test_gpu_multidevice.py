"""Kernel attributes are per device: the library must set them on every GPU it runs on.

cudaFuncSetAttribute (the dynamic shared-memory opt-in of the sweep, multigrid tail, ordered-sum and
convolution kernels) acts on the current device's context. The library keeps that set-up per device
ordinal, so a process that solves on device 0 and then on device 1 must get the same results on
both; the allocation-free ordered sum, whose scratch address is looked up per device, too. Needs two
GPUs (skipped otherwise).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import bit_equal, config_text, cuda_available, snapshot_config


def device_count() -> int:
    try:
        import torch
        return torch.cuda.device_count()
    except Exception:
        return 0


pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available() or device_count() < 2, reason="needs two CUDA devices")]


def test_solve_and_noalloc_sum_on_two_devices(sgpu_mod):
    import torch
    cfg = snapshot_config("short_16")
    cfg.update(N_cells_x="64", N_cells_y="48", momentum_solver="gs_multicolour", pressure_solver="mg",
               maxit="12", error_tolerance="0")
    values = np.random.default_rng(3).standard_normal((700, 300))
    want = sgpu_mod.ordered_sum(values)
    f = sgpu_mod.lib().sgpu_ordered_sum_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    results = []
    for dev in (0, 1):
        torch.cuda.set_device(dev)
        out = []
        for prec in ("fp64", "mixed"):
            with sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(dict(cfg, precision=prec)))) as s:
                _, log = s.run(12)
                out.append((log, s.download(0)))
        d_in = torch.from_numpy(values).to(f"cuda:{dev}")
        d_out = torch.zeros(1, dtype=torch.float64, device=f"cuda:{dev}")
        stream = torch.cuda.current_stream(dev)
        assert f(d_in.data_ptr(), 700, 300, 300, d_out.data_ptr(), stream.cuda_stream) == 0
        stream.synchronize()
        assert np.float64(d_out.item()).view(np.uint64) == np.float64(want).view(np.uint64)
        results.append(out)
    for (la, ua), (lb, ub) in zip(results[0], results[1]):
        assert bit_equal(la, lb) and bit_equal(ua, ub)
