"""Parity at the benchmark sizes.

* The plain FP64 method at 1024 x 1024 (Re 1000, QUICK / 4, gs_multicolour + mg V(2,2) down to 4 x 4),
  fixed work: error_tolerance = 0 and K = 50 outer iterations. The GPU's u, v, p, p' and residual log
  must equal the checker's bit for bit: the reference's own sources built in place (oracle/_ref,
  OpenMP on every host core) where present, else the C restatement (oracle/liborc.so). This is the
  fixed-work pattern of simple-hpc's GPU test (tests/hip/test_hip.cpp:166-174) at the size of the
  plain-method GPU configuration.
* The same at 4096 x 4096, K = 3: the size of the benchmark's FP64 arm.
* The mixed-precision solve at 1024 x 1024 after the same K = 50 iterations: u, v, p within 1e-6
  relative (max and L2) of the FP64 GPU run, the bound the mixed mode is held to at convergence.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bit_equal, config_text, cuda_available, describe_diff

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

FIELDS = (0, 1, 2, 27)  # u, v, p, p'


def cavity(n: int, k: int, **kw) -> dict:
    cfg = {"N_cells_x": n, "N_cells_y": n, "Re": 1000, "convection_scheme": "QUICK",
           "diffusion_order": 4, "momentum_solver": "gs_multicolour", "pressure_solver": "mg",
           "error_tolerance": 0, "maxit": k}
    cfg.update(kw)
    return cfg


def checker(sgpu_mod, oracle_mod, text: str):
    p = sgpu_mod.params_from_config(text)
    if oracle_mod.ref_available():
        return oracle_mod.Reference(text, p.shape), "reference (OpenMP)"
    return oracle_mod.Oracle(p), "C restatement"


def rel_errors(a: np.ndarray, b: np.ndarray) -> tuple[float, float]:
    return (float(np.max(np.abs(a - b)) / np.max(np.abs(b))),
            float(np.linalg.norm(a - b) / np.linalg.norm(b)))


@pytest.mark.parametrize("n,k", [(1024, 50), (4096, 3)])
def test_fp64_fixed_work_bit_exact_at_scale(sgpu_mod, oracle_mod, n, k):
    text = config_text(cavity(n, k))
    p = sgpu_mod.params_from_config(text)
    with sgpu_mod.Solver(p) as g:
        res, glog = g.run(k)
        assert res.iterations == k and not res.converged
        got = {f: g.download(f) for f in FIELDS}
    ref, kind = checker(sgpu_mod, oracle_mod, text)
    nr, conv, rlog = ref.run(k)
    print(f"{n}^2 x {k}: checked against the {kind}")
    assert nr == k
    assert bit_equal(glog, rlog), describe_diff(glog, rlog)
    for f in FIELDS:
        want = ref.get(f)
        assert bit_equal(got[f], want), f"field {f}: " + describe_diff(got[f], want)
    ref.close()


def test_mixed_close_to_fp64_at_1024(sgpu_mod):
    k = 50
    out = {}
    for prec in ("fp64", "mixed"):
        p = sgpu_mod.params_from_config(config_text(cavity(1024, k, precision=prec)))
        with sgpu_mod.Solver(p) as g:
            res, log = g.run(k)
            assert res.iterations == k
            out[prec] = ({f: g.download(f) for f in (0, 1, 2)}, log)
    for f, name in ((0, "u"), (1, "v"), (2, "p")):
        mx, l2 = rel_errors(out["mixed"][0][f], out["fp64"][0][f])
        print(f"{name}: max rel {mx:.3e}, L2 rel {l2:.3e}")
        assert mx < 1e-6 and l2 < 1e-6
    # the first iteration's momentum residuals precede every inner solve: FP64 to summation order
    a, b = out["mixed"][1][0, 1:3], out["fp64"][1][0, 1:3]
    assert np.all(np.abs(a - b) <= 1e-12 * np.abs(b))
