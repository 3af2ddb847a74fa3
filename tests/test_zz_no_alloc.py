"""sgpu_ordered_sum_noalloc: the ordered sum for callers that cannot allocate device memory.

The entry point keeps its scratch in a fixed device array inside the library and allocates nothing;
the caller passes device input and output. It must give exactly the sums of the allocating entry
point sgpu_ordered_sum (the tests of this repository compare sums bit for bit), on two calls in a
row — the second call reuses the shared scratch the first one left behind — and it must refuse
blocks larger than its fixed scratch with a clear message. This file is collected last so that a
run stopping at its first failure has already run every other test; it also passes on its own.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _noalloc(sgpu_mod):
    f = sgpu_mod.lib().sgpu_ordered_sum_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    return f


def _call(sgpu_mod, values: np.ndarray) -> float:
    import torch
    dev_in = torch.from_numpy(values).to("cuda")
    dev_out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _noalloc(sgpu_mod)(dev_in.data_ptr(), values.shape[0], values.shape[1], values.shape[1],
                            dev_out.data_ptr(), stream.cuda_stream)
    assert rc == 0, sgpu_mod.lib().sgpu_last_error().decode()
    stream.synchronize()
    return float(dev_out.cpu().item())


def test_noalloc_matches_allocating_sum_twice(sgpu_mod):
    rng = np.random.default_rng(20261203)
    first = rng.standard_normal((4101, 517)) * 10.0 ** rng.integers(-8, 8, (4101, 517))
    second = rng.standard_normal((333, 4099)) * 10.0 ** rng.integers(-8, 8, (333, 4099))
    for values in (first, second):
        got = _call(sgpu_mod, values)
        want = sgpu_mod.ordered_sum(values)
        assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (got, want)


def test_noalloc_rejects_oversized_blocks(sgpu_mod):
    import torch
    dev = torch.zeros((2, 4), dtype=torch.float64, device="cuda")
    out = torch.zeros((1,), dtype=torch.float64, device="cuda")
    rc = _noalloc(sgpu_mod)(dev.data_ptr(), 16385, 4, 4, out.data_ptr(), None)
    assert rc == sgpu_mod.E_INVALID
    assert "exceed the fixed scratch of 16384 rows" in sgpu_mod.lib().sgpu_last_error().decode()


def test_noalloc_strided_block_and_empty_shapes(sgpu_mod):
    """The two things this entry point adds over sgpu_ordered_sum: a row stride ld wider than the
    summed columns (a column slice of a wider device array), and empty blocks (sum 0.0)."""
    import torch
    rng = np.random.default_rng(7)
    wide = rng.standard_normal((1500, 700)) * 10.0 ** rng.integers(-6, 6, (1500, 700))
    dev = torch.from_numpy(wide).to("cuda")
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    f = _noalloc(sgpu_mod)
    stream = torch.cuda.current_stream()
    for c0, nc in ((0, 700), (13, 517), (699, 1), (250, 0)):
        rc = f(dev.data_ptr() + 8 * c0, 1500, nc, 700, out.data_ptr(), stream.cuda_stream)
        assert rc == 0, sgpu_mod.lib().sgpu_last_error().decode()
        stream.synchronize()
        got = float(out.cpu().item())
        want = sgpu_mod.ordered_sum(np.ascontiguousarray(wide[:, c0:c0 + nc])) if nc else 0.0
        assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (c0, nc, got, want)
    out.fill_(float("nan"))
    rc = f(dev.data_ptr(), 0, 700, 700, out.data_ptr(), stream.cuda_stream)
    assert rc == 0, sgpu_mod.lib().sgpu_last_error().decode()
    stream.synchronize()
    assert float(out.cpu().item()) == 0.0
    rc = f(dev.data_ptr(), 4, 8, 7, out.data_ptr(), stream.cuda_stream)  # ld < ncols
    assert rc == sgpu_mod.E_INVALID
