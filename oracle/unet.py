"""NumPy restatement of the learned warm-start network (forward pass, loss and
parameter gradients) for checking the library's CUDA implementation.

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of
stable_fluids_b200_network_{predict,gradients}; the product never imports it.

The reference has no learned warm start (it resets the pressure to zero every
step, backend-cuda.cu:644), so this oracle is pinned by its own gradient
check: analytic gradients against central finite differences in FP64
(tests/test_unet_oracle.py).

Two arithmetic modes:
  - bf16=False: plain FP64 everywhere (the mathematical network);
  - bf16=True : FP64 arithmetic, but every tensor the library stores in BF16
    (packed input, activations, pooled/upsampled tensors, weights, data
    gradients) is rounded to BF16 (round to nearest even) at the same points,
    so the library's results match to FP32-accumulation-order noise.

Layout: fields are (nz, ny, nx); activations (nz, ny, nx, C); weights
(27, cout, cin) with tap = (dz+1)*9 + (dy+1)*3 + (dx+1).
"""

from __future__ import annotations

import numpy as np

LAYERS = (
    ("enc0a", 16, 16), ("enc0b", 16, 16), ("enc1a", 16, 32), ("enc1b", 32, 32),
    ("bott_a", 32, 64), ("bott_b", 64, 64), ("dec1a", 96, 32), ("dec1b", 32, 32),
    ("dec0a", 48, 16), ("dec0b", 16, 16), ("out", 16, 16),
)


def split(flat):
    out, off = {}, 0
    for name, ci, co in LAYERS:
        wn = 27 * ci * co
        out[name] = (flat[off:off + wn].reshape(27, co, ci), flat[off + wn:off + wn + co])
        off += wn + co
    return out


def join(parts):
    return np.concatenate([np.concatenate([parts[n][0].ravel(), parts[n][1].ravel()]) for n, _, _ in LAYERS])


def bf16_round(x):
    """Round to BF16 (nearest even) through FP32, returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _taps():
    for tap in range(27):
        yield tap, tap // 9, (tap // 3) % 3, tap % 3


def conv(x, w, b=None):
    """3x3x3 convolution, zero padding: out[v, co] = b + sum w[tap, co, ci] x[v + off(tap), ci]."""
    nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((nz, ny, nx, w.shape[1]))
    for tap, dz, dy, dx in _taps():
        out += xp[dz:dz + nz, dy:dy + ny, dx:dx + nx, :] @ w[tap].T
    if b is not None:
        out += b
    return out


def conv_data_grad(g, w):
    """d/dx of conv: gx[v, ci] = sum_tap sum_co w[tap, co, ci] g[v - off(tap), co]."""
    nz, ny, nx, _ = g.shape
    gp = np.pad(g, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((nz, ny, nx, w.shape[2]))
    for tap, dz, dy, dx in _taps():
        out += gp[2 - dz:2 - dz + nz, 2 - dy:2 - dy + ny, 2 - dx:2 - dx + nx, :] @ w[tap]
    return out


def conv_weight_grad(x, g):
    """d/dw of conv: dw[tap, co, ci] = sum_v g[v, co] x[v + off(tap), ci]; db = sum_v g."""
    nz, ny, nx, cin = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    g2 = g.reshape(-1, g.shape[-1])
    dw = np.zeros((27, g.shape[-1], cin))
    for tap, dz, dy, dx in _taps():
        dw[tap] = g2.T @ xp[dz:dz + nz, dy:dy + ny, dx:dx + nx, :].reshape(-1, cin)
    return dw, g2.sum(axis=0)


def pool(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).mean(axis=(1, 3, 5))


def pool_grad(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 0), 2, 1), 2, 2) / 8.0


def upsample(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 0), 2, 1), 2, 2)


def upsample_grad(g):
    nz, ny, nx, c = g.shape
    return g.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).sum(axis=(1, 3, 5))


class UNet:
    def __init__(self, flat_params, bf16=False):
        self.p = split(np.asarray(flat_params, dtype=np.float64))
        self.bf16 = bf16
        self.r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
        # weights as the convolutions see them
        self.w = {n: self.r(self.p[n][0]) for n, _, _ in LAYERS}
        self.b = {n: self.p[n][1] for n, _, _ in LAYERS}

    def scale(self, b, h2):
        x = np.asarray(b, np.float64) * np.float64(np.float32(h2))
        rms = np.sqrt(np.sum(x * x) / x.size)
        s = 1.0 / rms if rms > 0 else 1.0
        return float(np.float32(s)) if self.bf16 else s

    def forward(self, b, p_prev, h2):
        r = self.r
        s = self.scale(b, h2)
        b = np.asarray(b, np.float64)
        p_prev = np.zeros_like(b) if p_prev is None else np.asarray(p_prev, np.float64)
        x = np.zeros(b.shape + (16,))
        if self.bf16:
            bs = (b.astype(np.float32) * np.float32(h2)).astype(np.float32) * np.float32(s)
            ps = p_prev.astype(np.float32) * np.float32(s)
            x[..., 0], x[..., 1] = r(bs), r(ps)
        else:
            x[..., 0], x[..., 1] = b * h2 * s, p_prev * s
        a = {"in": x}

        def layer(name, inp, relu=True):
            y = conv(inp, self.w[name], self.b[name])
            return r(np.maximum(y, 0.0)) if relu else y

        a["e0a"] = layer("enc0a", a["in"])
        a["e0b"] = layer("enc0b", a["e0a"])
        a["p0"] = r(pool(a["e0b"]))
        a["e1a"] = layer("enc1a", a["p0"])
        a["e1b"] = layer("enc1b", a["e1a"])
        a["p1"] = r(pool(a["e1b"]))
        a["ba"] = layer("bott_a", a["p1"])
        a["bb"] = layer("bott_b", a["ba"])
        a["cat1"] = np.concatenate([upsample(a["bb"]), a["e1b"]], axis=-1)
        a["d1a"] = layer("dec1a", a["cat1"])
        a["d1b"] = layer("dec1b", a["d1a"])
        a["cat0"] = np.concatenate([upsample(a["d1b"]), a["e0b"]], axis=-1)
        a["d0a"] = layer("dec0a", a["cat0"])
        a["d0b"] = layer("dec0b", a["d0a"])
        out = layer("out", a["d0b"], relu=False)[..., 0]
        if self.bf16:
            out = out.astype(np.float32).astype(np.float64)
        a["out"] = out
        a["scale"] = s
        a["p_prev"] = p_prev
        return a

    def predict(self, b, p_prev, h2):
        a = self.forward(b, p_prev, h2)
        return a["p_prev"] + a["out"] / a["scale"]

    def loss_and_gradients(self, b, p_prev, p_target, h2):
        """(loss, flat gradient) of mean((out - (p_target - p_prev) * scale)^2)."""
        r = self.r
        a = self.forward(b, p_prev, h2)
        s = a["scale"]
        target = (np.asarray(p_target, np.float64) - a["p_prev"]) * s
        if self.bf16:
            target = ((np.asarray(p_target, np.float32) - a["p_prev"].astype(np.float32)) * np.float32(s)).astype(np.float64)
        e = a["out"] - target
        n = e.size
        loss = float(np.sum(e * e) / n)
        g = np.zeros(e.shape + (16,))
        g[..., 0] = r(2.0 / n * e) if self.bf16 else 2.0 / n * e
        grads = {}

        def back(name, x_in, g_out, act=None, need_dx=True):
            """g_out: gradient at the layer output (post-ReLU mask applied by
            the caller); returns the data gradient of the layer input."""
            grads[name] = conv_weight_grad(x_in, g_out)
            return r(conv_data_grad(g_out, self.w[name])) if need_dx else None

        def relu_mask(g_, act):
            return np.where(act > 0, g_, 0.0)

        gd0b = back("out", a["d0b"], g)
        gd0b = relu_mask(gd0b, a["d0b"])
        gd0a = back("dec0b", a["d0a"], gd0b)
        gd0a = relu_mask(gd0a, a["d0a"])
        gcat0 = back("dec0a", a["cat0"], gd0a)
        gd1b = r(upsample_grad(gcat0[..., :32]))
        gd1b = relu_mask(gd1b, a["d1b"])
        gd1a = back("dec1b", a["d1a"], gd1b)
        gd1a = relu_mask(gd1a, a["d1a"])
        gcat1 = back("dec1a", a["cat1"], gd1a)
        gbb = r(upsample_grad(gcat1[..., :64]))
        gbb = relu_mask(gbb, a["bb"])
        gba = back("bott_b", a["ba"], gbb)
        gba = relu_mask(gba, a["ba"])
        gp1 = back("bott_a", a["p1"], gba)
        ge1b = r(gcat1[..., 64:] + pool_grad(gp1))
        ge1b = relu_mask(ge1b, a["e1b"])
        ge1a = back("enc1b", a["e1a"], ge1b)
        ge1a = relu_mask(ge1a, a["e1a"])
        gp0 = back("enc1a", a["p0"], ge1a)
        ge0b = r(gcat0[..., 32:] + pool_grad(gp0))
        ge0b = relu_mask(ge0b, a["e0b"])
        ge0a = back("enc0b", a["e0a"], ge0b)
        ge0a = relu_mask(ge0a, a["e0a"])
        back("enc0a", a["in"], ge0a, need_dx=False)
        return loss, join(grads)
