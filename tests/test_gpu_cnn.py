"""The learned warm start on the GPU: the network's kernels against the CPU oracle, its training, and
what the trained network gains the multigrid p' solve.

* forward output and loss/gradients of the BF16 tensor-core kernels against oracle/cnn_oracle.py
  (the same network in numpy with BF16 rounding at the same points; accumulation order differs, so
  the tolerance is a few BF16 ulps in relative L2);
* Adam training on the GPU lowers the loss; weights files round-trip;
* end to end: (b, converged p') pairs written by the solver itself train the network; attached to an
  unseen cavity, the warm-started multigrid (mg_mode = tolerance) meets the same tolerance in fewer
  V-cycles than from zero, and a useless network costs nothing in accuracy (the multigrid judges and
  discards its guess).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import config_text, cuda_available, snapshot_config

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def cnn_oracle():
    import cnn_oracle
    return cnn_oracle


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(np.asarray(b, np.float64)), 1e-30))


def test_forward_matches_oracle(sgpu_mod, cnn_oracle):
    params = cnn_oracle.init_params(16, 4, seed=11)
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 32, 48, 2)).astype(np.float32)
    with sgpu_mod.Cnn(16, 4) as net:
        assert net.num_params == params.size
        net.set_params(params)
        out = net.forward(x)
    ref, _ = cnn_oracle.UNetOracle(16, 4).forward(params, x)
    err = rel_l2(out, ref)
    print(f"forward relative L2 error vs oracle: {err:.2e}")
    assert err < 1e-2


def test_loss_and_gradients_match_oracle(sgpu_mod, cnn_oracle):
    """The 4-level network's loss and gradients against the oracle. The GPU accumulates in FP32 and
    the oracle in FP64, with BF16 rounding at the same points; a rounding that flips in one layer
    perturbs every layer after it, so over 28 BF16-rounded layers the gradients of two correct
    implementations lie a few percent apart. The oracle with FP32 accumulation against the oracle
    with FP64 accumulation shows that spread (1.2% over the whole vector, up to 3.7% per
    convolution); the GPU must stay within 5% per convolution and within twice that spread over the
    whole vector. The 1% per-convolution check of the kernels themselves is the shallow-network test
    below, where no cascade forms."""
    params = cnn_oracle.init_params(16, 4, seed=12)
    rng = np.random.default_rng(2)
    x = rng.normal(size=(2, 32, 32, 2)).astype(np.float32)
    t = rng.normal(size=(2, 32, 32)).astype(np.float32)
    with sgpu_mod.Cnn(16, 4) as net:
        net.set_params(params)
        loss, g = net.loss_grad(x, t)
    o = cnn_oracle.UNetOracle(16, 4)
    rloss, rg, _ = o.loss_grad(params, x, t)
    _, sg, _ = cnn_oracle.UNetOracle(16, 4, acc32=True).loss_grad(params, x, t)
    print(f"loss {loss:.6f} vs oracle {rloss:.6f}")
    assert abs(loss - rloss) <= 1e-2 * abs(rloss)
    for k, ((cin, cout, _), (wo, bo)) in enumerate(zip(o.convs, o.offs)):
        e = rel_l2(g[wo:bo + cout], rg[wo:bo + cout])
        spread = rel_l2(sg[wo:bo + cout], rg[wo:bo + cout])
        print(f"conv {k:2d} ({cin:3d} -> {cout:3d}): gradient relative L2 error {e:.2e}, "
              f"oracle FP32-vs-FP64 spread {spread:.2e}")
        assert e < 5e-2
    eh = rel_l2(g[o.head_w:], rg[o.head_w:])
    whole, whole_spread = rel_l2(g, rg), rel_l2(sg, rg)
    print(f"head: {eh:.2e}; whole vector: {whole:.2e} (oracle spread {whole_spread:.2e})")
    assert eh < 2e-2 and whole <= 2.0 * whole_spread + 5e-3


@pytest.mark.parametrize("base,levels", [(16, 1), (32, 1), (16, 2)])
def test_shallow_network_gradients_within_one_percent(sgpu_mod, cnn_oracle, base, levels):
    """Networks of 1 and 2 levels (2 and 6 convolutions): too shallow for rounding flips to cascade,
    so the tcgen05 forward, input-gradient and weight-gradient kernels must match the oracle's
    gradients to 1% per convolution (and the forward to 0.5%)."""
    params = cnn_oracle.init_params(base, levels, seed=31 + base + levels)
    rng = np.random.default_rng(7)
    x = rng.normal(size=(2, 24, 40, 2)).astype(np.float32)
    t = rng.normal(size=(2, 24, 40)).astype(np.float32)
    with sgpu_mod.Cnn(base, levels) as net:
        net.set_params(params)
        out = net.forward(x)
        loss, g = net.loss_grad(x, t)
    o = cnn_oracle.UNetOracle(base, levels)
    ref, _ = o.forward(params, x)
    rloss, rg, _ = o.loss_grad(params, x, t)
    ef = rel_l2(out, ref)
    print(f"base {base} levels {levels}: forward {ef:.2e}, loss {loss:.6f} vs {rloss:.6f}")
    assert ef < 5e-3
    for k, ((cin, cout, _), (wo, bo)) in enumerate(zip(o.convs, o.offs)):
        e = rel_l2(g[wo:bo + cout], rg[wo:bo + cout])
        print(f"conv {k} ({cin} -> {cout}): {e:.2e}")
        assert e < 1e-2


def test_training_lowers_loss_and_weights_round_trip(sgpu_mod, tmp_path):
    rng = np.random.default_rng(3)
    x = rng.normal(size=(8, 32, 32, 2)).astype(np.float32)
    # a smooth, learnable target: a local average of the first channel
    k = np.ones((5, 5)) / 25.0
    pad = np.pad(x[..., 0], ((0, 0), (2, 2), (2, 2)), mode="wrap")
    t = np.zeros_like(x[..., 0])
    for dy in range(5):
        for dx in range(5):
            t += k[dy, dx] * pad[:, dy:dy + 32, dx:dx + 32]
    with sgpu_mod.Cnn(16, 4, seed=4) as net:
        first = net.train_step(x, t, 1e-3)
        for _ in range(300):
            last = net.train_step(x, t, 1e-3)
        print(f"loss {first:.4f} -> {last:.4f}")
        assert last < 0.2 * first
        path = tmp_path / "w.unet"
        net.write(path)
        out = net.forward(x)
        with sgpu_mod.Cnn(path=path) as net2:
            assert np.array_equal(net2.params(), net.params())
            assert np.array_equal(net2.forward(x), out)
    with pytest.raises(sgpu_mod.SgpuError):
        sgpu_mod.Cnn(path=tmp_path / "missing.unet")
    with pytest.raises(sgpu_mod.SgpuError):
        with sgpu_mod.Cnn(16, 4) as net:
            net.forward(np.zeros((1, 12, 16, 2), np.float32))  # 12 is not a multiple of 8


def cavity(n: int, re: float, **kw) -> dict:
    cfg = snapshot_config("short_16")
    cfg.update(N_cells_x=str(n), N_cells_y=str(n), Re=str(re), convection_scheme="QUICK",
               diffusion_order="2", momentum_solver="gs_multicolour", pressure_solver="mg",
               error_tolerance="0", maxit="100000")
    cfg.update({k: str(v) for k, v in kw.items()})
    return cfg


def make_pairs(sgpu_mod, cases, iters, every, max_size):
    """(input, target) pairs written by the solver: FP64, p' solved to 1e-10 each iteration."""
    data = {}
    for n, re in cases:
        p = sgpu_mod.params_from_config(config_text(cavity(n, re, mg_mode="tolerance",
                                                           pressure_tolerance=1e-10, pressure_maxit=200)))
        with sgpu_mod.Solver(p) as s:
            for it in range(iters):
                s.outer_iteration()
                if it >= 2 and it % every == 0:
                    x, t, _ = s.cnn_sample(max_size)
                    data.setdefault(x.shape[:2], []).append((x, t))
    return data


def train(net, data, steps, batch, lr, rng):
    keys = sorted(data)
    losses = []
    for step in range(steps):
        key = keys[step % len(keys)]
        pool = data[key]
        idx = rng.integers(0, len(pool), min(batch, len(pool)))
        x = np.stack([pool[i][0] for i in idx])
        t = np.stack([pool[i][1] for i in idx])
        losses.append(net.train_step(x, t, lr))
    return losses


def vcycles(sgpu_mod, cfg, iters, net=None, max_size=32):
    p = sgpu_mod.params_from_config(config_text(cfg))
    with sgpu_mod.Solver(p) as s:
        if net is not None:
            s.attach_cnn(net, max_size)
        counts, rels = [], []
        for _ in range(iters):
            s.outer_iteration()
            st = s.last_solve_stats()
            counts.append(st["mg_vcycles"])
            rels.append(st["rel_residual"])
        fields = [s.download(f) for f in (0, 1, 2)]
        ws = s.warm_start_stats()
    return np.array(counts), np.array(rels), fields, ws


def test_trained_warm_start_saves_vcycles(sgpu_mod):
    max_size = 32
    data = make_pairs(sgpu_mod, [(64, 100), (64, 1000), (128, 400), (128, 2000), (96, 700)],
                      iters=80, every=2, max_size=max_size)
    npairs = sum(len(v) for v in data.values())
    print(f"{npairs} pairs, sizes {sorted(data)}")
    rng = np.random.default_rng(7)
    with sgpu_mod.Cnn(16, 4, seed=5) as net:
        losses = train(net, data, steps=600, batch=16, lr=2e-3, rng=rng)
        print(f"training loss {np.mean(losses[:20]):.4f} -> {np.mean(losses[-20:]):.4f}")
        assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:20])
        tol = 1e-6
        cfg = cavity(128, 1500, mg_mode="tolerance", pressure_tolerance=tol, pressure_maxit=100)
        iters = 30
        c0, r0, f0, _ = vcycles(sgpu_mod, cfg, iters)
        c1, r1, f1, ws = vcycles(sgpu_mod, cfg, iters, net, max_size)
    print(f"V-cycles per outer iteration: zero start {c0.mean():.2f}, warm start {c1.mean():.2f} "
          f"(warm starts {ws['used']}, discarded {ws['fallbacks']})")
    # the same tolerance is met either way
    assert (r0 <= tol).all() and (r1 <= tol).all()
    # the trained network's gain: fewer V-cycles to the same tolerance
    assert c1.mean() < c0.mean()
    # the fields agree to the accuracy the tolerance allows
    for a, b in zip(f1, f0):
        assert rel_l2(a, b) < 1e-4


def test_untrained_network_cannot_hurt_accuracy(sgpu_mod):
    tol = 1e-7
    cfg = cavity(96, 500, mg_mode="tolerance", pressure_tolerance=tol, pressure_maxit=100)
    with sgpu_mod.Cnn(16, 4, seed=9) as net:
        w = net.params()
        net.set_params(w * 50.0)  # a wildly wrong network
        c1, r1, f1, ws = vcycles(sgpu_mod, cfg, 8, net, 32)
    c0, r0, f0, _ = vcycles(sgpu_mod, cfg, 8)
    print(f"zero start {c0.tolist()}, bad network {c1.tolist()}, discarded {ws['fallbacks']}")
    assert ws["used"] == 8
    # every solve still meets the tolerance, so the fields agree to its accuracy
    assert (r1 <= tol).all()
    for a, b in zip(f1, f0):
        assert rel_l2(a, b) < 1e-4


def test_warm_start_mixed_precision_meets_tolerance(sgpu_mod):
    tol = 1e-5
    cfg = cavity(128, 1000, mg_mode="tolerance", pressure_tolerance=tol, pressure_maxit=100,
                 precision="mixed")
    with sgpu_mod.Cnn(16, 4, seed=2) as net:
        c, r, _, ws = vcycles(sgpu_mod, cfg, 5, net, 32)
    assert ws["used"] == 5 and (r <= tol).all()


def test_sample_rejects_mixed_precision(sgpu_mod):
    cfg = cavity(64, 100, precision="mixed")
    p = sgpu_mod.params_from_config(config_text(cfg))
    with sgpu_mod.Solver(p) as s:
        s.outer_iteration()
        with pytest.raises(sgpu_mod.SgpuError, match="fp64"):
            s.cnn_sample(32)
