"""CPU oracle of the warm-start U-Net (test infrastructure only: the product path never imports it).

The reference has no learned part, so this oracle is this project's own restatement of the network
the GPU library trains (simple-hpc_b200/csrc/cnn.cu): the same parameter layout, the same layers and
the same points where values are rounded to BF16, in numpy. Its backward pass is checked against
torch autograd in FP32 (tests/test_cnn_oracle.py); the GPU forward and gradients are checked against
it with BF16 rounding on (tests/test_gpu_cnn.py).

Layout (matches sgpu_cnn_get_params): per convolution W[cout][9][cin] then bias[cout], in network
order (encoder levels finest first, two convolutions each; decoder levels coarsest first); then the
head's `base` weights and its bias. Images are NHWC; the 2 input channels are zero-padded to 16.
"""
from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


class UNetOracle:
    """acc32: accumulate the convolutions in FP32 instead of FP64 (the same rounding points
    otherwise). The two variants differ only by FP32 rounding of the sums; the BF16 roundings that
    follow amplify that through the layers, which measures how far two correct implementations of
    this network can lie apart."""

    def __init__(self, base: int = 16, levels: int = 4, round_bf16: bool = True, acc32: bool = False):
        self.base, self.levels, self.rb = base, levels, round_bf16
        self.acc = np.float32 if acc32 else np.float64
        ch = lambda l: base << l  # noqa: E731
        convs = []
        for l in range(levels):
            convs.append((16 if l == 0 else ch(l - 1), ch(l), l))
            convs.append((ch(l), ch(l), l))
        for l in range(levels - 2, -1, -1):
            convs.append((ch(l + 1) + ch(l), ch(l), l))
            convs.append((ch(l), ch(l), l))
        self.convs = convs
        off, self.offs = 0, []
        for cin, cout, _ in convs:
            w_off = off
            off += cout * 9 * cin
            self.offs.append((w_off, off))
            off += cout
        self.head_w, self.head_b = off, off + base
        self.num_params = off + base + 1

    def _r(self, a):
        return bf16(a) if self.rb else np.asarray(a, np.float32)

    def unpack(self, params: np.ndarray):
        p = np.asarray(params, np.float32)
        Ws, bs = [], []
        for (cin, cout, _), (wo, bo) in zip(self.convs, self.offs):
            Ws.append(self._r(p[wo:wo + cout * 9 * cin].reshape(cout, 9, cin)))
            bs.append(p[bo:bo + cout])
        return Ws, bs, p[self.head_w:self.head_w + self.base], p[self.head_b]

    # ---- layers (float64 accumulation, rounded to FP32 then BF16 where the GPU stores BF16) ----
    @staticmethod
    def _shift(X, dy, dx):
        N, H, W, C = X.shape
        P = np.zeros((N, H + 2, W + 2, C), X.dtype)
        P[:, 1:H + 1, 1:W + 1] = X
        return P[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]

    def conv(self, X, Wt, b):
        N, H, W, _ = X.shape
        a = self.acc
        acc = np.zeros((N, H, W, Wt.shape[0]), a)
        for t in range(9):
            acc += self._shift(X, t // 3 - 1, t % 3 - 1).astype(a) @ Wt[:, t, :].T.astype(a)
        if b is not None:
            acc += b
        return acc.astype(np.float32)

    def conv_input_grad(self, dZ, Wt):
        N, H, W, _ = dZ.shape
        a = self.acc
        acc = np.zeros((N, H, W, Wt.shape[2]), a)
        for t in range(9):
            # dX[p + off(t)] += dZ[p] W[:, t, :]  ==  dX[q] += dZ[q - off(t)] W[:, t, :]
            acc += self._shift(dZ, -(t // 3 - 1), -(t % 3 - 1)).astype(a) @ Wt[:, t, :].astype(a)
        return acc.astype(np.float32)

    def conv_weight_grad(self, X, dZ):
        cout, cin = dZ.shape[3], X.shape[3]
        g = np.zeros((cout, 9, cin), np.float64)
        dz = dZ.reshape(-1, cout).astype(np.float64)
        for t in range(9):
            xs = self._shift(X, t // 3 - 1, t % 3 - 1).reshape(-1, cin).astype(np.float64)
            g[:, t, :] = dz.T @ xs
        return g

    @staticmethod
    def pool(X):
        N, H, W, C = X.shape
        return X.reshape(N, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4), dtype=np.float32) * np.float32(0.25)

    @staticmethod
    def up(X):
        return X.repeat(2, axis=1).repeat(2, axis=2)

    # ---- forward / backward ----
    def forward(self, params, x):
        """x: (n, h, w, 2). Returns (out (n, h, w), cache)."""
        Ws, bs, hw, hb = self.unpack(params)
        n, h, w, _ = x.shape
        X0 = np.zeros((n, h, w, 16), np.float32)
        X0[..., :2] = self._r(x)
        L, k = self.levels, 0
        ys, ins, pools, cats = [], [], {}, {}
        cur = X0
        for l in range(L):
            if l > 0:
                cur = self._r(self.pool(ys[k - 1]))
                pools[l] = cur
            for _ in range(2):
                ins.append(cur)
                cur = self._r(np.maximum(self.conv(cur, Ws[k], bs[k]), 0.0))
                ys.append(cur)
                k += 1
        for l in range(L - 2, -1, -1):
            cat = np.concatenate([self.up(cur), ys[2 * l + 1]], axis=3)
            cats[l] = cat
            cur = cat
            for _ in range(2):
                ins.append(cur)
                cur = self._r(np.maximum(self.conv(cur, Ws[k], bs[k]), 0.0))
                ys.append(cur)
                k += 1
        out = (cur.astype(np.float64) @ hw.astype(np.float64) + hb).astype(np.float32)
        return out, {"Ws": Ws, "ys": ys, "ins": ins, "hw": hw, "last": cur}

    def loss_grad(self, params, x, t):
        """Mean-squared error and its gradient (layout of the parameter vector)."""
        out, c = self.forward(params, x)
        Ws, ys, ins, hw = c["Ws"], c["ys"], c["ins"], c["hw"]
        npix = out.size
        diff = out.astype(np.float64) - t.astype(np.float64)
        loss = float(np.sum(diff * diff) / npix)
        d = (2.0 * diff / npix).astype(np.float32)
        g = np.zeros(self.num_params, np.float64)
        last = c["last"]
        g[self.head_w:self.head_w + self.base] = np.tensordot(d.astype(np.float64), last.astype(np.float64),
                                                              axes=([0, 1, 2], [0, 1, 2]))
        g[self.head_b] = float(np.sum(d, dtype=np.float64))
        L = self.levels
        K = len(self.convs)
        dys = [None] * K
        dys[K - 1] = self._r(d[..., None] * hw[None, None, None, :])

        def back(k, want_dx):
            cin, cout, _ = self.convs[k]
            dz = np.where(ys[k] > 0, dys[k], np.float32(0.0))
            wo, bo = self.offs[k]
            g[wo:wo + cout * 9 * cin] = self.conv_weight_grad(ins[k], dz).reshape(-1)
            g[bo:bo + cout] = dz.reshape(-1, cout).sum(axis=0, dtype=np.float64)
            return self._r(self.conv_input_grad(dz, Ws[k])) if want_dx else None

        k = K
        skip = {}
        for l in range(0, L - 1):
            k -= 2
            dys[k] = back(k + 1, True)
            dcat = back(k, True)
            ca = self.base << (l + 1)
            da = dcat[..., :ca]
            n_, H, W, _ = da.shape
            dys[k - 1] = self._r(da.reshape(n_, H // 2, 2, W // 2, 2, ca).sum(axis=(2, 4), dtype=np.float32))
            skip[l] = dcat[..., ca:]
        for l in range(L - 1, -1, -1):
            k -= 2
            if l < L - 1:
                dys[k + 1] = self._r(dys[k + 1] + skip[l])
            dys[k] = back(k + 1, True)
            dpool = back(k, l > 0)
            if l > 0:
                dys[k - 1] = self._r(np.float32(0.25) * self.up(dpool))
        return loss, g.astype(np.float32), out


def init_params(base: int = 16, levels: int = 4, seed: int = 0) -> np.ndarray:
    """Random parameters of the oracle's layout (He-like scale; padded input channels zero)."""
    o = UNetOracle(base, levels)
    rng = np.random.default_rng(seed)
    p = np.zeros(o.num_params, np.float32)
    for k, ((cin, cout, _), (wo, bo)) in enumerate(zip(o.convs, o.offs)):
        real = 2 if k == 0 else cin
        w = np.zeros((cout, 9, cin), np.float32)
        w[:, :, :real] = rng.normal(0.0, np.sqrt(2.0 / (9 * real)), (cout, 9, real))
        p[wo:wo + w.size] = w.reshape(-1)
        p[bo:bo + cout] = rng.normal(0.0, 0.05, cout)
    p[o.head_w:o.head_w + base] = rng.normal(0.0, np.sqrt(1.0 / base), base)
    p[o.head_b] = 0.1
    return p
