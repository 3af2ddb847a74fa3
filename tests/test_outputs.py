"""Output files: byte-identical to the reference's write_outputs (src/io.cpp:43-151).

The field CSVs, centrelines and alog.csv are compared byte for byte with the files the reference's
own writer produces for the same state (oracle/_ref); timing.csv and run_info.json carry run-specific
values (times, git hash, compiler), so their structure and keys are compared. The CLI test runs the
`simple` driver on the GPU and checks its files against the oracle's state.
"""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO, bit_equal, config_text, cuda_available, snapshot_config

FIELD_FILES = ["u.csv", "v.csv", "p.csv", "ux_centre.csv", "uy_centre.csv", "alog.csv"]


def _state(sgpu_mod, oracle_mod, cfg, iters):
    p = sgpu_mod.params_from_config(config_text(cfg))
    o = oracle_mod.Oracle(p)
    n, conv, log = o.run(iters)
    return p, o, log


@pytest.mark.parametrize("nx,ny", [(16, 16), (32, 40), (7, 3)])
def test_writer_matches_reference_bytes(sgpu_mod, oracle_mod, tmp_path, nx, ny):
    if not oracle_mod.ref_available():
        pytest.skip("reference build not present")
    cfg = snapshot_config("short_16")
    cfg.update(N_cells_x=str(nx), N_cells_y=str(ny), maxit="6")
    p, o, log = _state(sgpu_mod, oracle_mod, cfg, 6)
    ours = tmp_path / "ours"
    p.output_dir = str(ours).encode()
    sgpu_mod.write_outputs(p, o.get(0), o.get(1), o.get(2), log)
    ref = oracle_mod.Reference(config_text(cfg), p.shape)
    for f in (0, 1, 2):
        ref.set(f, o.get(f))
    theirs = tmp_path / "theirs"
    assert oracle_mod.ref_lib().ref_write_outputs(ref._h, str(theirs).encode(), log.shape[0],
                                                  log.ctypes.data_as(__import__("ctypes").POINTER(
                                                      __import__("ctypes").c_double))) == 0
    for name in FIELD_FILES:
        assert (ours / name).read_bytes() == (theirs / name).read_bytes(), name
    a = [ln.split(",")[0] for ln in (ours / "timing.csv").read_text().splitlines()]
    b = [ln.split(",")[0] for ln in (theirs / "timing.csv").read_text().splitlines()]
    assert a == b
    ka = list(json.loads((ours / "run_info.json").read_text()).keys())
    kb = list(json.loads((theirs / "run_info.json").read_text()).keys())
    assert ka == kb


def test_write_fields_false_skips_fields(sgpu_mod, oracle_mod, tmp_path):
    cfg = snapshot_config("short_16")
    cfg.update(write_fields="False", maxit="2")
    p, o, log = _state(sgpu_mod, oracle_mod, cfg, 2)
    p.output_dir = str(tmp_path).encode()
    sgpu_mod.write_outputs(p, o.get(0), o.get(1), o.get(2), log)
    names = sorted(x.name for x in tmp_path.iterdir())
    assert names == ["alog.csv", "run_info.json", "timing.csv"]


def test_cli_usage_and_errors(tmp_path):
    exe = REPO / "simple-hpc_b200" / "simple"
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr == "usage: simple <config>\n"
    bad = tmp_path / "bad.cfg"
    bad.write_text("N_cells_x = 8\nN_cells_x = 9\n")
    r = subprocess.run([str(exe), str(bad)], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stderr == "error (rank 0): config line 2: duplicate key 'N_cells_x'\n"


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_cli_gpu_run_writes_reference_outputs(sgpu_mod, oracle_mod, tmp_path):
    cfg = snapshot_config("converged_32x40")
    cfg.update(momentum_solver="gs_multicolour", pressure_solver="mg", backend="gpu",
               output_dir=str(tmp_path / "out"))
    cfg_path = tmp_path / "run.cfg"
    cfg_path.write_text(config_text(cfg))
    exe = REPO / "simple-hpc_b200" / "simple"
    r = subprocess.run([str(exe), str(cfg_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "gpu: " in r.stdout and "iter 1  res_u" in r.stdout
    p, o, log = _state(sgpu_mod, oracle_mod, cfg, int(cfg["maxit"]))
    last = r.stdout.strip().splitlines()[-1]
    assert last.startswith(f"converged after {log.shape[0]} iterations in ")
    ref_dir = tmp_path / "oracle_out"
    p.output_dir = str(ref_dir).encode()
    sgpu_mod.write_outputs(p, o.get(0), o.get(1), o.get(2), log)
    for name in FIELD_FILES:
        assert (tmp_path / "out" / name).read_bytes() == (ref_dir / name).read_bytes(), name
    info = json.loads((tmp_path / "out" / "run_info.json").read_text())
    assert info["backend"] == "gpu" and info["iterations"] == log.shape[0] and info["converged"]


def test_restart_files_round_trip(sgpu_mod, tmp_path):
    """restart_from reads back exactly the u.csv, v.csv, p.csv the writer writes (%.18e)."""
    cfg = snapshot_config("short_16")
    cfg["output_dir"] = str(tmp_path / "run")
    p = sgpu_mod.params_from_config(config_text(cfg))
    rng = np.random.default_rng(4)
    u, v, pf = (rng.normal(size=(p.nrows, p.ncols)) * 10.0 ** rng.integers(-300, 300, (p.nrows, p.ncols))
                for _ in range(3))
    u[0, 0], v[1, 1], pf[2, 2] = -0.0, 5e-324, -1.7976931348623157e308
    sgpu_mod.write_outputs(p, u, v, pf, np.zeros((1, 4)))
    ru, rv, rp = sgpu_mod.read_fields(p, tmp_path / "run")
    for a, b in ((ru, u), (rv, v), (rp, pf)):
        assert a.view(np.uint64).tolist() == b.view(np.uint64).tolist()
    # a grid of another size, a missing file and a damaged value are errors naming the file
    cfg2 = dict(cfg, N_cells_x="20")
    p2 = sgpu_mod.params_from_config(config_text(cfg2))
    with pytest.raises(sgpu_mod.SgpuError, match="u.csv has"):
        sgpu_mod.read_fields(p2, tmp_path / "run")
    with pytest.raises(sgpu_mod.SgpuError, match="cannot read"):
        sgpu_mod.read_fields(p, tmp_path / "nowhere")
    f = tmp_path / "run" / "v.csv"
    f.write_text(f.read_text().replace(",", ",x", 1))
    with pytest.raises(sgpu_mod.SgpuError, match="v.csv row 1"):
        sgpu_mod.read_fields(p, tmp_path / "run")


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_restart_continues_the_run(sgpu_mod, tmp_path):
    """10 iterations, written out, then 10 more from restart_from: the fields of 20 straight."""
    base = snapshot_config("converged_32x40")
    base.update(momentum_solver="gs_multicolour", pressure_solver="mg", error_tolerance="0")
    p = sgpu_mod.params_from_config(config_text(dict(base, output_dir=str(tmp_path / "a"))))
    with sgpu_mod.Solver(p) as s:
        res, log = s.run(10)
        f10 = [s.download(k) for k in (0, 1, 2)]
    sgpu_mod.write_outputs(p, *f10, log, res)
    p2 = sgpu_mod.params_from_config(config_text(dict(base, restart_from=str(tmp_path / "a"))))
    assert p2.restart_from.decode() == str(tmp_path / "a")
    u, v, pf = sgpu_mod.read_fields(p2, p2.restart_from.decode())
    with sgpu_mod.Solver(p2, u, v, pf) as s:
        s.run(10)
        restarted = [s.download(k) for k in (0, 1, 2)]
    with sgpu_mod.Solver(p) as s:
        s.run(20)
        straight = [s.download(k) for k in (0, 1, 2)]
    for a, b in zip(restarted, straight):
        assert bit_equal(a, b)
