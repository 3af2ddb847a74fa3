"""The warm-start network's CPU oracle (oracle/cnn_oracle.py) against torch autograd, on the CPU.

The reference has no learned part, so the oracle that the GPU kernels are checked against is this
project's own numpy restatement. These tests pin it: with BF16 rounding off, its loss and every
parameter gradient must equal torch's (FP64 autograd of the same network, the parameters loaded from
the same vector); its BF16 rounding must equal torch's float32 -> bfloat16 conversion.
"""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
F = torch.nn.functional

from cnn_oracle import UNetOracle, bf16, init_params  # noqa: E402


def torch_unet_loss(o: UNetOracle, params: np.ndarray, x: np.ndarray, t: np.ndarray):
    """The same U-Net in torch (NCHW, FP64); returns (loss, gradient vector)."""
    p = torch.tensor(params.astype(np.float64), requires_grad=True)
    n, h, w, _ = x.shape
    X = torch.zeros((n, 16, h, w), dtype=torch.float64)
    X[:, :2] = torch.tensor(x.astype(np.float64)).permute(0, 3, 1, 2)

    def conv(k, inp):
        cin, cout, _ = o.convs[k]
        wo, bo = o.offs[k]
        W = p[wo:wo + cout * 9 * cin].reshape(cout, 9, cin).permute(0, 2, 1).reshape(cout, cin, 3, 3)
        return F.relu(F.conv2d(inp, W, p[bo:bo + cout], padding=1))

    L, k, ys, cur = o.levels, 0, [], X
    for lv in range(L):
        if lv > 0:
            cur = F.avg_pool2d(ys[-1], 2)
        for _ in range(2):
            cur = conv(k, cur)
            ys.append(cur)
            k += 1
    for lv in range(L - 2, -1, -1):
        cur = torch.cat([F.interpolate(cur, scale_factor=2, mode="nearest"), ys[2 * lv + 1]], dim=1)
        for _ in range(2):
            cur = conv(k, cur)
            k += 1
    hw = p[o.head_w:o.head_w + o.base]
    out = torch.einsum("nchw,c->nhw", cur, hw) + p[o.head_b]
    loss = torch.mean((out - torch.tensor(t.astype(np.float64))) ** 2)
    loss.backward()
    return float(loss.detach()), p.grad.numpy(), out.detach().numpy()


@pytest.mark.parametrize("base,levels,h,w", [(16, 4, 16, 24), (16, 3, 8, 12)])
def test_oracle_matches_torch_autograd(base, levels, h, w):
    o = UNetOracle(base, levels, round_bf16=False)
    params = init_params(base, levels, seed=3)
    rng = np.random.default_rng(5)
    x = rng.normal(size=(2, h, w, 2)).astype(np.float32)
    t = rng.normal(size=(2, h, w)).astype(np.float32)
    loss, g, out = o.loss_grad(params, x, t)
    tl, tg, tout = torch_unet_loss(o, params, x, t)
    np.testing.assert_allclose(out, tout, rtol=1e-4, atol=1e-5)
    assert abs(loss - tl) <= 1e-5 * abs(tl)
    # every parameter block (the oracle keeps activations in FP32: agreement to ~1e-6 relative)
    for k, ((cin, cout, _), (wo, bo)) in enumerate(zip(o.convs, o.offs)):
        a, b = g[wo:bo + cout], tg[wo:bo + cout]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 1e-4, f"conv {k}: relative gradient error {rel:.2e}"
    head = slice(o.head_w, o.num_params)
    np.testing.assert_allclose(g[head], tg[head], rtol=1e-4, atol=1e-7)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.normal(size=10000).astype(np.float32) * np.float32(10.0) ** rng.integers(-8, 8, 10000),
                           np.array([0.0, -0.0, 1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, 65504.0,
                                     np.finfo(np.float32).tiny, 3.0e38], np.float32)])
    ours = bf16(vals)
    ref = torch.tensor(vals).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))


def test_parameter_count_and_flops_layout():
    o = UNetOracle(16, 4)
    # conv weights + biases for 14 convolutions, head 16 + 1
    expect = 0
    for cin, cout, _ in o.convs:
        expect += cout * 9 * cin + cout
    assert o.num_params == expect + 17
    assert len(o.convs) == 4 * 4 - 2
