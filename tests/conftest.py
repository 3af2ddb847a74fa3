"""Shared test setup.

Markers: ``gpu`` tests need a CUDA device and run the B200 solver through its C ABI; everything
else runs on the CPU (the oracle against the golden fixtures, the parser, the C-ABI symbol table).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
sys.path.insert(0, str(REPO / "simple-hpc_b200"))
sys.path.insert(0, str(REPO / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def config_text(cfg: dict) -> str:
    return "\n".join(f"{k} = {v}" for k, v in cfg.items()) + "\n"


def load_golden(name: str) -> dict:
    d = np.load(GOLDEN / name, allow_pickle=False)
    out = {k: d[k] for k in d.files}
    out["config"] = json.loads(str(out["config"]))
    return out


# The reference's snapshot configurations (configs/snapshot/*.cfg in simple-hpc), as stored in the
# golden fixtures; tests derive their cases from these by overriding keys.
def snapshot_config(name: str) -> dict:
    return dict(load_golden(f"snapshot_{name}.npz")["config"])


@pytest.fixture(scope="session")
def sgpu_mod():
    import sgpu
    sgpu.lib()
    return sgpu


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.orc_lib()
    return oracle


def bit_equal(a: np.ndarray, b: np.ndarray) -> bool:
    """Equal bit for bit (distinguishes -0.0 from 0.0, NaN payloads compare equal)."""
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def describe_diff(a: np.ndarray, b: np.ndarray) -> str:
    if a.shape != b.shape:
        return f"shape {a.shape} != {b.shape}"
    neq = a.view(np.uint64) != b.view(np.uint64)
    if not neq.any():
        return "identical"
    idx = np.argwhere(neq)
    i, j = idx[0]
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    return (f"{neq.sum()} cells differ; first at ({i},{j}): {a[i, j]!r} vs {b[i, j]!r}; "
            f"max rel {np.nanmax(rel):.3e}")
