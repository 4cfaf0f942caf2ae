"""CPU oracle of the learned gradient preconditioner's U-Net (test
infrastructure: only tests and the benchmark's CPU leg use it).

numpy restatement of the network, its loss and its backward pass with the
GPU path's rounding points: activations and activation gradients rounded to
BF16 (round to nearest even) where the GPU stores them, conv weights used in
BF16, the head's weights and every bias in FP32; sums in FP64 (the GPU sums
in FP32 on the tensor cores, so results agree to BF16 rounding, not bit for
bit). With ``bf16=False`` nothing is rounded and the backward pass is the
exact gradient of the FP64 forward (checked against finite differences).

The network (no reference counterpart): 4 resolution levels with base, 2x,
4x, 8x base channels; two 3x3 conv + ReLU per level; 2x2 mean pooling down;
nearest upsampling and concatenation with the skip tensor up; 1x1 head to
one output channel. Input channels are zero-padded to 16.
"""
import numpy as np


def layer_table(base=32):
    """[(name, cin, cout)] of the 3x3 convolutions in parameter order."""
    c1, c2, c3, c4 = base, 2 * base, 4 * base, 8 * base
    return [("enc1a", 16, c1), ("enc1b", c1, c1), ("enc2a", c1, c2), ("enc2b", c2, c2),
            ("enc3a", c2, c3), ("enc3b", c3, c3), ("bota", c3, c4), ("botb", c4, c4),
            ("dec3a", c3 + c4, c3), ("dec3b", c3, c3), ("dec2a", c2 + c3, c2), ("dec2b", c2, c2),
            ("dec1a", c1 + c2, c1), ("dec1b", c1, c1)]


def bf16(x):
    """Round float32 values to BF16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).reshape(np.shape(x))


def unflatten(p, base=32):
    """Flat FP32 parameter vector -> {name: (w [9, cout, cin], b [cout])} + head."""
    out, o = {}, 0
    for name, cin, cout in layer_table(base):
        w = p[o:o + 9 * cout * cin].reshape(9, cout, cin)
        o += 9 * cout * cin
        out[name] = (w, p[o:o + cout])
        o += cout
    out["head"] = (p[o:o + base], p[o + base:o + base + 1])
    o += base + 1
    assert o == len(p)
    return out


def n_params(base=32):
    return sum(9 * ci * co + co for _, ci, co in layer_table(base)) + base + 1


class Net:
    def __init__(self, params, base=32, bf16_round=True):
        self.base = base
        self.P = unflatten(np.asarray(params, np.float32), base)
        self.r = bf16 if bf16_round else (lambda a: np.asarray(a, np.float64))

    # ---- primitives -------------------------------------------------------
    def _w(self, name):
        w = self.P[name][0]
        return self.r(w).astype(np.float64)

    @staticmethod
    def _shift(x, dy, dx):
        """x padded by one (zeros), window for tap (dy, dx) in 0..2."""
        N, H, W, C = x.shape
        xp = np.zeros((N, H + 2, W + 2, C))
        xp[:, 1:-1, 1:-1] = x
        return xp[:, dy:dy + H, dx:dx + W]

    def conv(self, x, w):
        """sum_tap x(p + tap) @ w[tap].T, FP64; w [9, cout, cin]."""
        N, H, W, _ = x.shape
        y = np.zeros((N, H, W, w.shape[1]))
        for tap in range(9):
            y += self._shift(x, tap // 3, tap % 3) @ w[tap].T
        return y

    def conv_relu(self, x, name):
        w, b = self.P[name]
        return self.r(np.maximum(self.conv(x, self._w(name)) + b.astype(np.float64), 0.0))

    def pool(self, x):
        s = x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2]
        return self.r(0.25 * s)

    @staticmethod
    def up(x):
        return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)

    # ---- network ------------------------------------------------------------
    def forward(self, x):
        """x [N, H, W, cin<=16] -> (out [N, H, W], cache)."""
        N, H, W, cin = x.shape
        x16 = np.zeros((N, H, W, 16))
        x16[..., :cin] = self.r(np.asarray(x, np.float32))
        c = {"x": x16}
        c["e1a"] = self.conv_relu(x16, "enc1a")
        c["e1"] = self.conv_relu(c["e1a"], "enc1b")
        c["p1"] = self.pool(c["e1"])
        c["e2a"] = self.conv_relu(c["p1"], "enc2a")
        c["e2"] = self.conv_relu(c["e2a"], "enc2b")
        c["p2"] = self.pool(c["e2"])
        c["e3a"] = self.conv_relu(c["p2"], "enc3a")
        c["e3"] = self.conv_relu(c["e3a"], "enc3b")
        c["p3"] = self.pool(c["e3"])
        c["ba"] = self.conv_relu(c["p3"], "bota")
        c["b"] = self.conv_relu(c["ba"], "botb")
        c["c3"] = np.concatenate([c["e3"], self.up(c["b"])], axis=-1)
        c["d3a"] = self.conv_relu(c["c3"], "dec3a")
        c["d3"] = self.conv_relu(c["d3a"], "dec3b")
        c["c2"] = np.concatenate([c["e2"], self.up(c["d3"])], axis=-1)
        c["d2a"] = self.conv_relu(c["c2"], "dec2a")
        c["d2"] = self.conv_relu(c["d2a"], "dec2b")
        c["c1"] = np.concatenate([c["e1"], self.up(c["d2"])], axis=-1)
        c["d1a"] = self.conv_relu(c["c1"], "dec1a")
        c["d1"] = self.conv_relu(c["d1a"], "dec1b")
        wh, bh = self.P["head"]
        out = c["d1"] @ wh.astype(np.float64) + float(bh[0])
        return out, c

    # ---- backward -----------------------------------------------------------
    def _wgrad(self, x, dz):
        """dw [9, cout, cin] = sum_p dz[p] x[p + tap]^T."""
        cin, cout = x.shape[-1], dz.shape[-1]
        dzf = dz.reshape(-1, cout)
        return np.stack([dzf.T @ self._shift(x, t // 3, t % 3).reshape(-1, cin) for t in range(9)])

    def _dgrad(self, dz, name):
        """input gradient of a conv: sum_tap dz(p - tap) w[tap]."""
        w = self._w(name)
        wb = np.stack([w[8 - t].T for t in range(9)])  # [9, cin, cout]: the flipped transpose
        return self.conv(dz, wb)

    def backward(self, cache, dout):
        """Gradients of sum(dout * out) w.r.t. every parameter: {name: (dw, db)}."""
        c, r, g = cache, self.r, {}
        wh, _ = self.P["head"]
        d = np.asarray(dout, np.float64)
        g["head"] = (np.einsum("nhw,nhwc->c", d, c["d1"]), np.array([d.sum()]))
        dz = r(d[..., None] * wh.astype(np.float64) * (c["d1"] > 0))

        def conv_back(name, x, dz, masks=None, split=None):
            g[name] = (self._wgrad(x, dz), dz.reshape(-1, dz.shape[-1]).sum(0))
            if masks is None:
                return None
            dx = self._dgrad(dz, name)
            if split is None:
                return r(dx * (masks > 0)) if masks is not False else r(dx)
            a = dx[..., :split]
            b = dx[..., split:]
            m0, m1 = masks
            return (r(a * (m0 > 0)) if m0 is not None else r(a), r(b * (m1 > 0)) if m1 is not None else r(b))

        def up_back(du, x):
            s = du[:, 0::2, 0::2] + du[:, 0::2, 1::2] + du[:, 1::2, 0::2] + du[:, 1::2, 1::2]
            return r(s * (x > 0))

        def pool_back(dp, x, dx):
            return r(dx + 0.25 * self.up(dp) * (x > 0))

        b1, b2, b3 = self.base, 2 * self.base, 4 * self.base
        dz = conv_back("dec1b", c["d1a"], dz, c["d1a"])
        de1, du1 = conv_back("dec1a", c["c1"], dz, (c["e1"], None), split=b1)
        dz = up_back(du1, c["d2"])
        dz = conv_back("dec2b", c["d2a"], dz, c["d2a"])
        de2, du2 = conv_back("dec2a", c["c2"], dz, (c["e2"], None), split=b2)
        dz = up_back(du2, c["d3"])
        dz = conv_back("dec3b", c["d3a"], dz, c["d3a"])
        de3, du3 = conv_back("dec3a", c["c3"], dz, (c["e3"], None), split=b3)
        dz = up_back(du3, c["b"])
        dz = conv_back("botb", c["ba"], dz, c["ba"])
        dp3 = conv_back("bota", c["p3"], dz, False)
        de3 = pool_back(dp3, c["e3"], de3)
        dz = conv_back("enc3b", c["e3a"], de3, c["e3a"])
        dp2 = conv_back("enc3a", c["p2"], dz, False)
        de2 = pool_back(dp2, c["e2"], de2)
        dz = conv_back("enc2b", c["e2a"], de2, c["e2a"])
        dp1 = conv_back("enc2a", c["p1"], dz, False)
        de1 = pool_back(dp1, c["e1"], de1)
        dz = conv_back("enc1b", c["e1a"], de1, c["e1a"])
        conv_back("enc1a", c["x"], dz, None)
        return g

    def flat_grad(self, g):
        parts = []
        for name, _, _ in layer_table(self.base):
            parts += [g[name][0].ravel(), g[name][1].ravel()]
        parts += [g["head"][0].ravel(), g["head"][1].ravel()]
        return np.concatenate(parts)


def mse_loss(out, target, weight=None, inv_norm=None):
    """(loss, dout) of sum w (out - target)^2 * inv_norm."""
    d = np.asarray(out, np.float64) - np.asarray(target, np.float64)
    w = 1.0 if weight is None else np.asarray(weight, np.float64)
    if inv_norm is None:
        inv_norm = 1.0 / d.size
    return float(np.sum(w * d * d) * inv_norm), 2.0 * w * d * inv_norm


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One bias-corrected Adam step in place (FP64 restatement)."""
    g = g + wd * p
    m[:] = b1 * m + (1 - b1) * g
    v[:] = b2 * v + (1 - b2) * g * g
    p -= lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p
