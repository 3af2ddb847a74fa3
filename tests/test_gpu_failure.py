"""Device-side failure detection, tested without a GPU fault.

The mixed mode's correction sweep waits on mbarriers for the record copies it issues. Every such wait
is bounded: one that runs out sets a device word, which sgpu_run and sgpu_batch_run report as
SGPU_E_TIMEOUT, instead of hanging the GPU. sgpu_selftest_bounded_wait runs that same wait helper
on an mbarrier that nothing ever completes. The wait must give up and say so, and the context must
stay usable: a solve right after it runs normally.
"""
from __future__ import annotations

import pytest

from conftest import config_text, cuda_available, snapshot_config


@pytest.mark.parametrize("polls", [1, 4096])
@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_bounded_wait_gives_up_and_reports(sgpu_mod, polls):
    assert sgpu_mod.selftest_bounded_wait(polls)


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_context_usable_after_a_give_up(sgpu_mod):
    assert sgpu_mod.selftest_bounded_wait(4096)
    cfg = snapshot_config("short_16")
    cfg.update(N_cells_x="48", N_cells_y="48", momentum_solver="gs_multicolour", pressure_solver="mg",
               precision="mixed", maxit="5", error_tolerance="0")
    with sgpu_mod.Solver(sgpu_mod.params_from_config(config_text(cfg))) as s:
        res, log = s.run(5)
    assert res.iterations == 5 and log.shape[0] == 5


def test_selftest_rejects_bad_arguments(sgpu_mod):
    # checked before any device work, so this runs without a GPU
    for polls in (0, -3, (1 << 20) + 1):
        with pytest.raises(sgpu_mod.SgpuError, match="polls"):
            sgpu_mod.selftest_bounded_wait(polls)
