"""CPU tests of the U-Net oracle: its backward pass is the exact gradient of
its FP64 forward (central finite differences along per-layer directions), its
BF16 rounding is round-to-nearest-even, and its layer table is the product's."""
import numpy as np

import unet_oracle as uo


def test_bf16_rounding_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 1e-30], np.float32)
    r = uo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                    # tie -> even
    assert r[2] == np.float32(1.0 + 2 ** -6)  # tie -> even (up)
    assert r[3] == -2.5 and r[4] == 0.0
    assert abs(r[5] - 1e-30) / 1e-30 < 2 ** -8


def test_layer_tables_agree():
    from otfwi_b200.unet import layer_table
    for base in (4, 32):
        assert layer_table(base) == uo.layer_table(base)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    base = 4
    n = uo.n_params(base)
    p = rng.standard_normal(n) * 0.3
    x = rng.standard_normal((2, 8, 8, 3))
    t = rng.standard_normal((2, 8, 8))

    def net(pp):
        m = uo.Net(pp.astype(np.float32), base, bf16_round=False)
        m.P = uo.unflatten(pp, base)  # FP64 parameters
        return m

    m = net(p)
    out, cache = m.forward(x)
    _, dout = uo.mse_loss(out, t)
    g = m.flat_grad(m.backward(cache, dout))

    def loss(pp):
        return uo.mse_loss(net(pp).forward(x)[0], t)[0]

    errs = []
    o = 0
    for name, cin, cout in uo.layer_table(base) + [("head", base, 1)]:
        sz = 9 * cin * cout + cout if name != "head" else base + 1
        v = np.zeros(n)
        v[o:o + sz] = rng.standard_normal(sz)
        eps = 1e-6
        fd = (loss(p + eps * v) - loss(p - eps * v)) / (2 * eps)
        errs.append(abs(fd - g @ v) / abs(fd))
        o += sz
    errs = np.array(errs)
    # ReLU kinks on the 1x1 bottleneck of an 8x8 input can cost a few 1e-4
    assert np.median(errs) < 1e-7
    assert errs.max() < 5e-3


def test_oracle_adam_first_step_is_sign_times_lr():
    p = np.array([1.0, -2.0, 0.5])
    g = np.array([0.3, -1e-3, 0.0])
    m, v = np.zeros(3), np.zeros(3)
    uo.adam(p, g, m, v, 1, lr=0.1, eps=0.0 + 1e-12)
    assert np.allclose(p, [0.9, -1.9, 0.5])
