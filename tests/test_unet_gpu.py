"""GPU tests of the U-Net kernels against the numpy oracle: one fused
convolution (two inputs, upsampled second input, bias, ReLU, split masked
outputs), its weight gradient, the whole network's output and parameter
gradients, one Adam step, and a training run that must cut the loss.

Tolerances: the GPU sums in FP32 on the tensor cores and the oracle in FP64,
both from the same BF16 operands, so outputs agree to BF16 rounding
(relative L2 <= 1e-2; measured values are printed)."""
import numpy as np
import pytest

import unet_oracle as uo

pytestmark = pytest.mark.gpu


def _bf(a):
    import torch
    return torch.as_tensor(uo.bf16(np.asarray(a, np.float32))).to(torch.bfloat16).cuda().contiguous()


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


def test_fused_conv_and_weight_gradient(lib):
    import torch
    from otfwi_b200.unet import UNet, _declare, _p
    L = _declare(lib)
    rng = np.random.default_rng(3)
    N, H, W, c0, c1, cout, split = 2, 24, 40, 32, 64, 64, 32
    x0 = rng.standard_normal((N, H, W, c0))
    x1 = rng.standard_normal((N, H // 2, W // 2, c1))
    w = rng.standard_normal((9, cout, c0 + c1)) * 0.05
    b = rng.standard_normal(cout).astype(np.float32)
    m0 = np.maximum(rng.standard_normal((N, H, W, split)), 0)
    X0, X1, Wt = _bf(x0), _bf(x1), _bf(w.reshape(-1))
    M0 = _bf(m0)
    B = torch.as_tensor(b).cuda()
    D0 = torch.empty((N, H, W, split), dtype=torch.bfloat16, device="cuda")
    D1 = torch.empty((N, H, W, cout - split), dtype=torch.bfloat16, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert L.otf_unet_conv3x3(_p(X0), c0, _p(X1), c1, 1, _p(Wt), _p(B), 1, _p(D0), _p(M0), _p(D1), None,
                              split, cout, N, H, W, st) == 0
    torch.cuda.synchronize()
    net = uo.Net(np.zeros(uo.n_params(4), np.float32), 4)
    xin = np.concatenate([_np(X0), net.up(_np(X1))], axis=-1)
    ref = np.maximum(net.conv(xin, _np(Wt).reshape(9, cout, c0 + c1)) + b, 0)
    r0 = _rel(_np(D0), ref[..., :split] * (m0 > 0))
    r1 = _rel(_np(D1), ref[..., split:])
    print("conv rel L2", r0, r1)
    assert r0 <= 1e-2 and r1 <= 1e-2
    # weight gradient of the same convolution for a seeded dz
    dz = rng.standard_normal((N, H, W, cout))
    DZ = _bf(dz)
    dW = torch.zeros(9 * cout * (c0 + c1), dtype=torch.float32, device="cuda")
    sm = torch.cuda.get_device_properties(0).multi_processor_count
    assert L.otf_unet_conv3x3_wgrad(_p(X0), c0, _p(X1), c1, 1, _p(DZ), cout, _p(dW), N, H, W, sm, st) == 0
    torch.cuda.synchronize()
    refw = net._wgrad(xin, _np(DZ))
    rw = _rel(dW.cpu().numpy().reshape(9, cout, c0 + c1), refw)
    print("wgrad rel L2", rw)
    assert rw <= 1e-4  # FP32 vs FP64 sums of the same BF16 products


def _net_case(N=2, H=32, W=48, seed=5):
    from otfwi_b200.unet import UNet
    rng = np.random.default_rng(seed)
    net = UNet(base=32, in_ch=3, seed=seed)
    x = rng.standard_normal((N, H, W, 3)).astype(np.float32)
    t = (0.05 * rng.standard_normal((N, H, W))).astype(np.float32)
    return net, x, t


def test_network_forward_and_gradients_vs_oracle(lib):
    """Forward output against the oracle's forward; parameter gradients
    against the oracle's backward run on the GPU's own activations (so only
    the backward arithmetic is compared, relative L2 <= 1e-2 per layer), and
    end to end against the oracle's own forward + backward, where BF16
    rounding differences of the two forward passes compound with depth
    (relative L2 <= 8e-2 per layer)."""
    import torch
    net, x, t = _net_case()
    # make the head non-trivial so every layer's gradient is well scaled
    o = net.head_off
    p = net.state()
    p[o:o + 32] = np.random.default_rng(1).standard_normal(32).astype(np.float32) * 0.2
    net.params.copy_(torch.as_tensor(p))
    net.pack()
    X = torch.as_tensor(x).cuda()
    T = torch.as_tensor(t).cuda()
    out = net.forward(X)
    loss = net.loss_grad(T)
    N, H, W = t.shape
    B = net._buffers(N, H, W)
    net.backward(B["dout"])
    torch.cuda.synchronize()
    ora = uo.Net(p, 32)
    oo, cache = ora.forward(x)
    lo, dout = uo.mse_loss(oo, t)
    rel_out = _rel(out.cpu().numpy(), oo)
    print("output rel L2", rel_out, "loss", float(loss), lo)
    assert rel_out <= 1e-2
    assert abs(float(loss) - lo) <= 1e-2 * lo
    got = net.grads.cpu().numpy()
    # the GPU's activations as the oracle's cache
    gc = {k: _np(B[k]) for k in ("x", "e1a", "e1", "p1", "e2a", "e2", "p2", "e3a", "e3", "p3", "ba", "b",
                                 "d3a", "d3", "d2a", "d2", "d1a", "d1")}
    gc["c3"] = np.concatenate([gc["e3"], ora.up(gc["b"])], axis=-1)
    gc["c2"] = np.concatenate([gc["e2"], ora.up(gc["d3"])], axis=-1)
    gc["c1"] = np.concatenate([gc["e1"], ora.up(gc["d2"])], axis=-1)
    for label, g, tol in (("same activations", ora.backward(gc, B["dout"].cpu().numpy().astype(np.float64)), 1e-2),
                          ("end to end", ora.backward(cache, dout), 8e-2)):
        worst, per = 0.0, {}
        for name, cin, cout in uo.layer_table(32):
            a, b = net.offsets[name]
            rw = _rel(got[a:b], g[name][0].ravel())
            rb = _rel(got[b:b + cout], g[name][1])
            per[name] = (f"{rw:.1e}", f"{rb:.1e}")
            worst = max(worst, rw, rb)
        rh = _rel(got[net.head_off:net.head_off + 33], np.concatenate([g["head"][0], g["head"][1]]))
        print(label, "worst layer rel L2", worst, "head", rh, "per layer (weights, bias)", per)
        assert worst <= tol and rh <= tol


def test_adam_step_matches_oracle(lib):
    import torch
    net, _, _ = _net_case()
    rng = np.random.default_rng(9)
    g = rng.standard_normal(net.n_params).astype(np.float32)
    p0 = net.state().astype(np.float64)
    net.grads.copy_(torch.as_tensor(g))
    net.adam(lr=1e-3)
    net.grads.copy_(torch.as_tensor(0.5 * g))
    net.adam(lr=1e-3)
    m, v = np.zeros_like(p0), np.zeros_like(p0)
    uo.adam(p0, g.astype(np.float64), m, v, 1, 1e-3)
    uo.adam(p0, 0.5 * g.astype(np.float64), m, v, 2, 1e-3)
    assert np.max(np.abs(net.state() - p0)) <= 1e-6


def test_training_cuts_the_loss(lib):
    """A smooth seeded mapping (target = local mean of channel 0 minus channel
    1) is learned: 150 Adam steps cut the loss at least 5x."""
    import torch
    from otfwi_b200.unet import UNet
    rng = np.random.default_rng(0)
    N, H, W = 8, 32, 32
    x = rng.standard_normal((N, H, W, 3)).astype(np.float32)
    k = np.ones((5, 5)) / 25
    from numpy.lib.stride_tricks import sliding_window_view
    pad = np.pad(x[..., 0], ((0, 0), (2, 2), (2, 2)))
    t = (sliding_window_view(pad, (5, 5), axis=(1, 2)) * k).sum((-1, -2)) - 0.3 * x[..., 1]
    net = UNet(base=32, in_ch=3, seed=1)
    X = torch.as_tensor(x).cuda()
    T = torch.as_tensor(t.astype(np.float32)).cuda()
    losses = []
    for s in range(150):
        losses.append(float(net.train_step(X, T, lr=2e-3)))
    print("loss first/last", losses[0], losses[-1])
    assert losses[-1] < losses[0] / 5
