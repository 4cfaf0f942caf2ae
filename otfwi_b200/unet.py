"""BF16 U-Net of the learned gradient preconditioner, run and trained on the
GPU by the library's own kernels (otf_unet_*, unet.cu).

No reference counterpart: the reference inverts with plain L-BFGS-B on the
raw gradient (regression.py:82-88). The network maps per-cell features
(gradient, illumination, current model; normalised) to a model update. 4
resolution levels with base, 2x, 4x, 8x base channels, two 3x3 conv + ReLU
per level, 2x2 mean pooling, nearest upsampling + skip concatenation, a 1x1
head. Activations BF16 [N][H][W][C]; FP32 master weights, gradients and Adam
moments; PyTorch only allocates device memory and supplies the stream.
"""
import ctypes
from ctypes import c_float, c_int, c_longlong, c_void_p

import numpy as np

from . import _lib


def layer_table(base=32):
    """[(name, cin, cout)] of the 3x3 convolutions in parameter order."""
    c1, c2, c3, c4 = base, 2 * base, 4 * base, 8 * base
    return [("enc1a", 16, c1), ("enc1b", c1, c1), ("enc2a", c1, c2), ("enc2b", c2, c2),
            ("enc3a", c2, c3), ("enc3b", c3, c3), ("bota", c3, c4), ("botb", c4, c4),
            ("dec3a", c3 + c4, c3), ("dec3b", c3, c3), ("dec2a", c2 + c3, c2), ("dec2b", c2, c2),
            ("dec1a", c1 + c2, c1), ("dec1b", c1, c1)]


def _declare(L):
    if getattr(L, "_unet_declared", False):
        return L
    v, i, f, ll = c_void_p, c_int, c_float, c_longlong
    sig = {
        "otf_unet_conv3x3": [v, i, v, i, i, v, v, i, v, v, v, v, i, i, i, i, i, v],
        "otf_unet_conv3x3_packed": [v, i, v, i, i, v, v, v, i, v, v, v, v, i, i, i, i, i, v],
        "otf_unet_pack_weights_tc": [v, i, i, v, v],
        "otf_unet_conv3x3_wgrad": [v, i, v, i, i, v, i, v, i, i, i, i, v],
        "otf_unet_bias_grad": [v, i, ll, v, v],
        "otf_unet_pool2": [v, v, i, i, i, i, v],
        "otf_unet_pool2_bwd": [v, v, v, i, i, i, i, v],
        "otf_unet_up2_bwd": [v, v, v, i, i, i, i, v],
        "otf_unet_pack_input": [v, i, ll, v, v],
        "otf_unet_head": [v, v, v, ll, v, v],
        "otf_unet_head_bwd": [v, v, v, ll, v, v, v, v],
        "otf_unet_mse": [v, v, v, ll, f, v, v, v],
        "otf_unet_adam": [v, v, v, v, ll, f, f, f, f, i, f, v],
        "otf_unet_pack_weights": [v, i, i, v, v, v],
        "otf_unet_set_umma": [i],
        "otf_unet_status": [],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.restype = c_int
        fn.argtypes = args
    L._unet_declared = True
    return L


def _p(t):
    return None if t is None else c_void_p(t.data_ptr())


class UNet:
    """The preconditioner network on one GPU.

    ``forward(x)``: x [N, H, W, cin] FP32 CUDA tensor (cin <= 16, H and W
    multiples of 8) -> [N, H, W] FP32. ``train_step(x, target, weight)``: one
    Adam step on the weighted mean squared error; returns the loss as a
    device tensor (no synchronisation)."""

    def __init__(self, base=32, in_ch=3, seed=0, params=None, lib=None, device="cuda"):
        import torch
        self.torch = torch
        self.L = _declare(_lib.load(lib))
        if base != 32:
            raise ValueError("the head kernels are built for 32 base channels")
        self.base, self.in_ch, self.dev = base, in_ch, torch.device(device)
        self.layers = layer_table(base)
        self.offsets = {}
        o = 0
        for name, cin, cout in self.layers:
            self.offsets[name] = (o, o + 9 * cin * cout)
            o += 9 * cin * cout + cout
        self.head_off = o
        self.n_params = o + base + 1
        if params is None:
            params = self.init_params(seed)
        self.params = torch.as_tensor(np.asarray(params, np.float32)).to(self.dev).contiguous()
        assert self.params.numel() == self.n_params
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self.wf, self.wb = {}, {}
        self.wfp, self.wbp = {}, {}  # the same, packed for the tcgen05 kernels' bulk copies
        for name, cin, cout in self.layers:
            self.wf[name] = torch.empty(9 * cout * cin, dtype=torch.bfloat16, device=self.dev)
            self.wb[name] = torch.empty(9 * cout * cin, dtype=torch.bfloat16, device=self.dev)
            self.wfp[name] = torch.empty(9 * cout * cin, dtype=torch.bfloat16, device=self.dev)
            self.wbp[name] = torch.empty(9 * cout * cin, dtype=torch.bfloat16, device=self.dev)
        self.sm = torch.cuda.get_device_properties(self.dev).multi_processor_count
        self._bufs = {}
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.pack()

    # ---- parameters -------------------------------------------------------
    def init_params(self, seed):
        """He-normal conv weights (input channels beyond in_ch zero), zero
        biases, a small head."""
        rng = np.random.default_rng(seed)
        out = []
        for name, cin, cout in self.layers:
            fan = 9 * (self.in_ch if name == "enc1a" else cin)
            w = rng.standard_normal((9, cout, cin)) * np.sqrt(2.0 / fan)
            if name == "enc1a":
                w[:, :, self.in_ch:] = 0.0
            out += [w.ravel(), np.zeros(cout)]
        out += [rng.standard_normal(self.base) * 0.01 / np.sqrt(self.base), np.zeros(1)]
        return np.concatenate(out).astype(np.float32)

    def weight(self, name):
        a, b = self.offsets[name]
        return self.params[a:b]

    def bias(self, name):
        _, cin, cout = next(l for l in self.layers if l[0] == name)
        b = self.offsets[name][1]
        return self.params[b:b + cout]

    def _stream(self):
        return c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _ok(self, rc):
        if rc != 0:
            _lib.check(self.L)
            raise _lib.OtfwiError("unet kernel failed")

    def pack(self):
        """BF16 forward and input-gradient copies of every conv weight, and
        both regrouped by 8-channel plane for the tcgen05 kernels."""
        st = self._stream()
        for name, cin, cout in self.layers:
            self._ok(self.L.otf_unet_pack_weights(_p(self.weight(name)), cout, cin, _p(self.wf[name]),
                                                  _p(self.wb[name]), st))
            self._ok(self.L.otf_unet_pack_weights_tc(_p(self.wf[name]), cout, cin, _p(self.wfp[name]), st))
            self._ok(self.L.otf_unet_pack_weights_tc(_p(self.wb[name]), cin, cout, _p(self.wbp[name]), st))

    def state(self):
        return self.params.detach().cpu().numpy().copy()

    def save(self, path):
        np.savez(path, params=self.state(), base=self.base, in_ch=self.in_ch)

    @classmethod
    def load(cls, path, **kw):
        d = np.load(path)
        return cls(base=int(d["base"]), in_ch=int(d["in_ch"]), params=d["params"], **kw)

    # ---- buffers ----------------------------------------------------------
    def _buffers(self, N, H, W):
        key = (N, H, W)
        if key in self._bufs:
            return self._bufs[key]
        torch = self.torch
        if H % 8 or W % 8:
            raise ValueError("U-Net input height and width must be multiples of 8")
        b1, b2, b3, b4 = self.base, 2 * self.base, 4 * self.base, 8 * self.base
        shapes = {"x": (1, 16), "e1a": (1, b1), "e1": (1, b1), "p1": (2, b1), "e2a": (2, b2), "e2": (2, b2),
                  "p2": (4, b2), "e3a": (4, b3), "e3": (4, b3), "p3": (8, b3), "ba": (8, b4), "b": (8, b4),
                  "d3a": (4, b3), "d3": (4, b3), "d2a": (2, b2), "d2": (2, b2), "d1a": (1, b1), "d1": (1, b1)}
        B = {}
        for k, (s, c) in shapes.items():
            B[k] = torch.empty((N, H // s, W // s, c), dtype=torch.bfloat16, device=self.dev)
        # gradients: one per forward tensor that needs one, plus temporaries
        for k, (s, c) in shapes.items():
            if k != "x":
                B["g_" + k] = torch.empty((N, H // s, W // s, c), dtype=torch.bfloat16, device=self.dev)
        B["g_u1"] = torch.empty((N, H, W, b2), dtype=torch.bfloat16, device=self.dev)
        B["g_u2"] = torch.empty((N, H // 2, W // 2, b3), dtype=torch.bfloat16, device=self.dev)
        B["g_u3"] = torch.empty((N, H // 4, W // 4, b4), dtype=torch.bfloat16, device=self.dev)
        B["out"] = torch.empty((N, H, W), dtype=torch.float32, device=self.dev)
        B["dout"] = torch.empty((N, H, W), dtype=torch.float32, device=self.dev)
        self._bufs[key] = B
        return B

    # ---- primitives -------------------------------------------------------
    # optional per-launch timing of the convolutions: a list that receives
    # (kind, layer, flop, start event, end event) per call, or None
    timers = None

    def _timed(self, kind, name, flop, launch):
        if self.timers is None:
            return launch()
        import torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream(self.dev)  # the stream the kernels are launched on (_stream)
        e0.record(st)
        rc = launch()
        e1.record(st)
        self.timers.append((kind, name, flop, e0, e1))
        return rc

    def _conv(self, name, src0, dst, N, H, W, src1=None, up1=0, relu=1):
        _, cin, cout = next(l for l in self.layers if l[0] == name)
        c0 = src0.shape[-1]
        c1 = 0 if src1 is None else src1.shape[-1]
        assert c0 + c1 == cin
        self._ok(self._timed("fwd", name, 18.0 * cin * cout * N * H * W, lambda: self.L.otf_unet_conv3x3_packed(
            _p(src0), c0, _p(src1), c1, up1, _p(self.wf[name]), _p(self.wfp[name]), _p(self.bias(name)), relu,
            _p(dst), None, None, None, cout, cout, N, H, W, self._stream())))

    def _dgrad(self, name, dz, dst0, mask0, N, H, W, dst1=None, split=None):
        """input gradient of conv `name` from its pre-activation gradient dz."""
        _, cin, cout = next(l for l in self.layers if l[0] == name)
        split = cin if split is None else split
        self._ok(self._timed("dgrad", name, 18.0 * cin * cout * N * H * W, lambda: self.L.otf_unet_conv3x3_packed(
            _p(dz), cout, None, 0, 0, _p(self.wb[name]), _p(self.wbp[name]), None, 0, _p(dst0), _p(mask0),
            _p(dst1), None, split, cin, N, H, W, self._stream())))

    def _wgrad(self, name, src0, dz, N, H, W, src1=None, up1=0):
        _, cin, cout = next(l for l in self.layers if l[0] == name)
        c0 = src0.shape[-1]
        c1 = 0 if src1 is None else src1.shape[-1]
        a, b = self.offsets[name]
        st = self._stream()
        self._ok(self._timed("wgrad", name, 18.0 * cin * cout * N * H * W, lambda: self.L.otf_unet_conv3x3_wgrad(
            _p(src0), c0, _p(src1), c1, up1, _p(dz), cout, _p(self.grads[a:b]), N, H, W, self.sm, st)))
        self._ok(self.L.otf_unet_bias_grad(_p(dz), cout, N * H * W, _p(self.grads[b:b + cout]), st))

    # ---- network ----------------------------------------------------------
    def forward(self, x):
        """x [N, H, W, cin] FP32 CUDA -> [N, H, W] FP32 (a view of an internal buffer)."""
        torch = self.torch
        N, H, W, cin = x.shape
        assert cin <= 16 and x.dtype == torch.float32 and x.is_contiguous()
        B = self._buffers(N, H, W)
        st = self._stream()
        self._ok(self.L.otf_unet_pack_input(_p(x), cin, N * H * W, _p(B["x"]), st))
        H2, W2, H4, W4, H8, W8 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        self._conv("enc1a", B["x"], B["e1a"], N, H, W)
        self._conv("enc1b", B["e1a"], B["e1"], N, H, W)
        self._ok(self.L.otf_unet_pool2(_p(B["e1"]), _p(B["p1"]), N, H, W, self.base, st))
        self._conv("enc2a", B["p1"], B["e2a"], N, H2, W2)
        self._conv("enc2b", B["e2a"], B["e2"], N, H2, W2)
        self._ok(self.L.otf_unet_pool2(_p(B["e2"]), _p(B["p2"]), N, H2, W2, 2 * self.base, st))
        self._conv("enc3a", B["p2"], B["e3a"], N, H4, W4)
        self._conv("enc3b", B["e3a"], B["e3"], N, H4, W4)
        self._ok(self.L.otf_unet_pool2(_p(B["e3"]), _p(B["p3"]), N, H4, W4, 4 * self.base, st))
        self._conv("bota", B["p3"], B["ba"], N, H8, W8)
        self._conv("botb", B["ba"], B["b"], N, H8, W8)
        self._conv("dec3a", B["e3"], B["d3a"], N, H4, W4, src1=B["b"], up1=1)
        self._conv("dec3b", B["d3a"], B["d3"], N, H4, W4)
        self._conv("dec2a", B["e2"], B["d2a"], N, H2, W2, src1=B["d3"], up1=1)
        self._conv("dec2b", B["d2a"], B["d2"], N, H2, W2)
        self._conv("dec1a", B["e1"], B["d1a"], N, H, W, src1=B["d2"], up1=1)
        self._conv("dec1b", B["d1a"], B["d1"], N, H, W)
        o = self.head_off
        self._ok(self.L.otf_unet_head(_p(B["d1"]), _p(self.params[o:o + self.base]),
                                      _p(self.params[o + self.base:o + self.base + 1]), N * H * W, _p(B["out"]),
                                      st))
        return B["out"]

    def backward(self, dout):
        """Parameter gradients (into self.grads, zeroed first) of sum(dout *
        out) for the last forward; dout [N, H, W] FP32 CUDA."""
        N, H, W = dout.shape
        B = self._buffers(N, H, W)
        st = self._stream()
        self.grads.zero_()
        b1, b2, b3, b4 = self.base, 2 * self.base, 4 * self.base, 8 * self.base
        H2, W2, H4, W4, H8, W8 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        o = self.head_off
        self._ok(self.L.otf_unet_head_bwd(_p(B["d1"]), _p(self.params[o:o + b1]), _p(dout), N * H * W,
                                          _p(B["g_d1"]), _p(self.grads[o:o + b1]),
                                          _p(self.grads[o + b1:o + b1 + 1]), st))
        # decoder, level 1
        self._wgrad("dec1b", B["d1a"], B["g_d1"], N, H, W)
        self._dgrad("dec1b", B["g_d1"], B["g_d1a"], B["d1a"], N, H, W)
        self._wgrad("dec1a", B["e1"], B["g_d1a"], N, H, W, src1=B["d2"], up1=1)
        self._dgrad("dec1a", B["g_d1a"], B["g_e1"], B["e1"], N, H, W, dst1=B["g_u1"], split=b1)
        self._ok(self.L.otf_unet_up2_bwd(_p(B["g_u1"]), _p(B["d2"]), _p(B["g_d2"]), N, H2, W2, b2, st))
        # level 2
        self._wgrad("dec2b", B["d2a"], B["g_d2"], N, H2, W2)
        self._dgrad("dec2b", B["g_d2"], B["g_d2a"], B["d2a"], N, H2, W2)
        self._wgrad("dec2a", B["e2"], B["g_d2a"], N, H2, W2, src1=B["d3"], up1=1)
        self._dgrad("dec2a", B["g_d2a"], B["g_e2"], B["e2"], N, H2, W2, dst1=B["g_u2"], split=b2)
        self._ok(self.L.otf_unet_up2_bwd(_p(B["g_u2"]), _p(B["d3"]), _p(B["g_d3"]), N, H4, W4, b3, st))
        # level 3
        self._wgrad("dec3b", B["d3a"], B["g_d3"], N, H4, W4)
        self._dgrad("dec3b", B["g_d3"], B["g_d3a"], B["d3a"], N, H4, W4)
        self._wgrad("dec3a", B["e3"], B["g_d3a"], N, H4, W4, src1=B["b"], up1=1)
        self._dgrad("dec3a", B["g_d3a"], B["g_e3"], B["e3"], N, H4, W4, dst1=B["g_u3"], split=b3)
        self._ok(self.L.otf_unet_up2_bwd(_p(B["g_u3"]), _p(B["b"]), _p(B["g_b"]), N, H8, W8, b4, st))
        # bottleneck
        self._wgrad("botb", B["ba"], B["g_b"], N, H8, W8)
        self._dgrad("botb", B["g_b"], B["g_ba"], B["ba"], N, H8, W8)
        self._wgrad("bota", B["p3"], B["g_ba"], N, H8, W8)
        self._dgrad("bota", B["g_ba"], B["g_p3"], None, N, H8, W8)
        self._ok(self.L.otf_unet_pool2_bwd(_p(B["g_p3"]), _p(B["e3"]), _p(B["g_e3"]), N, H4, W4, b3, st))
        # encoder
        self._wgrad("enc3b", B["e3a"], B["g_e3"], N, H4, W4)
        self._dgrad("enc3b", B["g_e3"], B["g_e3a"], B["e3a"], N, H4, W4)
        self._wgrad("enc3a", B["p2"], B["g_e3a"], N, H4, W4)
        self._dgrad("enc3a", B["g_e3a"], B["g_p2"], None, N, H4, W4)
        self._ok(self.L.otf_unet_pool2_bwd(_p(B["g_p2"]), _p(B["e2"]), _p(B["g_e2"]), N, H2, W2, b2, st))
        self._wgrad("enc2b", B["e2a"], B["g_e2"], N, H2, W2)
        self._dgrad("enc2b", B["g_e2"], B["g_e2a"], B["e2a"], N, H2, W2)
        self._wgrad("enc2a", B["p1"], B["g_e2a"], N, H2, W2)
        self._dgrad("enc2a", B["g_e2a"], B["g_p1"], None, N, H2, W2)
        self._ok(self.L.otf_unet_pool2_bwd(_p(B["g_p1"]), _p(B["e1"]), _p(B["g_e1"]), N, H, W, b1, st))
        self._wgrad("enc1b", B["e1a"], B["g_e1"], N, H, W)
        self._dgrad("enc1b", B["g_e1"], B["g_e1a"], B["e1a"], N, H, W)
        self._wgrad("enc1a", B["x"], B["g_e1a"], N, H, W)
        return self.grads

    def loss_grad(self, target, weight=None, inv_norm=None):
        """Weighted MSE of the last forward output; fills its gradient. Returns the loss (device)."""
        N, H, W = target.shape
        B = self._buffers(N, H, W)
        n = N * H * W
        inv = float(1.0 / n if inv_norm is None else inv_norm)
        self.loss.zero_()
        self._ok(self.L.otf_unet_mse(_p(B["out"]), _p(target), _p(weight), n, inv, _p(B["dout"]),
                                     _p(self.loss), self._stream()))
        return self.loss

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, weight_decay=0.0):
        self.step_count += 1
        self._ok(self.L.otf_unet_adam(_p(self.params), _p(self.grads), _p(self.m), _p(self.v), self.n_params,
                                      lr, b1, b2, eps, self.step_count, weight_decay, self._stream()))
        self.pack()

    def train_step(self, x, target, weight=None, lr=1e-3):
        self.forward(x)
        loss = self.loss_grad(target, weight).clone()
        N, H, W = target.shape
        self.backward(self._buffers(N, H, W)["dout"])
        self.adam(lr)
        return loss


def _bench_conv(a):
    """One forward convolution (bias + ReLU) of the given shape, with the
    weights packed as the network passes them, launched `iters` times after 3
    warm-up launches, timed with CUDA events."""
    import json

    import torch
    N, H, W, cin, cout = (int(v) for v in a.conv.split(","))
    L = _declare(_lib.load())
    L.otf_unet_set_umma(0 if a.legacy else 1)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.randn(N, H, W, cin, device="cuda", generator=g).to(torch.bfloat16)
    w = (torch.randn(9 * cout * cin, device="cuda", generator=g) / (3.0 * cin ** 0.5)).to(torch.bfloat16)
    b = torch.zeros(cout, device="cuda")
    y = torch.empty(N, H, W, cout, dtype=torch.bfloat16, device="cuda")
    st = c_void_p(torch.cuda.current_stream().cuda_stream)
    wp = torch.empty_like(w)  # packed once, as the network packs after each update
    if L.otf_unet_pack_weights_tc(_p(w), cout, cin, _p(wp), st) != 0:
        _lib.check(L)

    def launch():
        if L.otf_unet_conv3x3_packed(_p(x), cin, None, 0, 0, _p(w), _p(wp), _p(b), 1, _p(y), None, None, None,
                                     cout, cout, N, H, W, st) != 0:
            _lib.check(L)

    for _ in range(3):
        launch()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.iters):
        launch()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.iters
    flop = 18.0 * cin * cout * N * H * W
    print(json.dumps({"conv": [N, H, W, cin, cout], "kernel": "mma.sync" if a.legacy else "tcgen05",
                      "ms": ms, "tflops": flop / ms / 1e9, "device_status": int(L.otf_unet_status())}))


def _bench(argv=None):
    """Time forward and training steps: python -m otfwi_b200.unet --n 16 --hw 256."""
    import argparse
    import json

    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=16)
    ap.add_argument("--hw", type=int, default=256)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--legacy", action="store_true", help="warp-level mma.sync convolutions instead of tcgen05")
    ap.add_argument("--tcgen05-all", action="store_true",
                    help="tcgen05 for every layer's weight gradient too (by default small layers keep mma.sync)")
    ap.add_argument("--convs", action="store_true",
                    help="also time every 3x3 convolution launch of a training step (forward, input gradient, "
                         "weight gradient) and report TFLOP/s per kind and per layer")
    ap.add_argument("--conv", default="",
                    help="time one forward 3x3 convolution alone instead of the network: N,H,W,cin,cout")
    a = ap.parse_args(argv)
    if a.conv:
        return _bench_conv(a)
    net = UNet(base=32)
    net.L.otf_unet_set_umma(0 if a.legacy else (2 if a.tcgen05_all else 1))
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.randn(a.n, a.hw, a.hw, 3, device="cuda", generator=g)
    t = 0.01 * torch.randn(a.n, a.hw, a.hw, device="cuda", generator=g)
    for _ in range(3):
        net.train_step(x, t)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.iters):
        net.forward(x)
    e1.record()
    torch.cuda.synchronize()
    f_ms = e0.elapsed_time(e1) / a.iters
    e0.record()
    for _ in range(a.iters):
        net.train_step(x, t)
    e1.record()
    torch.cuda.synchronize()
    s_ms = e0.elapsed_time(e1) / a.iters
    # 3x3 convolution FLOPs of one forward (2 per multiply-add); pooling,
    # head and elementwise work excluded
    flop = 0.0
    for name, cin, cout in net.layers:
        lvl = {"enc1": 0, "dec1": 0, "enc2": 1, "dec2": 1, "enc3": 2, "dec3": 2, "bota": 3, "botb": 3}[name[:4]]
        flop += 2.0 * 9 * cin * cout * a.n * (a.hw >> lvl) ** 2
    out = {"n": a.n, "hw": a.hw, "conv": "mma.sync" if a.legacy else ("tcgen05 (all)" if a.tcgen05_all else "tcgen05"),
           "forward_ms": f_ms, "forward_tflops": flop / f_ms / 1e9,
           "train_step_ms": s_ms, "train_tflops": 3 * flop / s_ms / 1e9}
    if a.convs:
        # per-launch events around each convolution of a few training steps
        # (the launches run back to back, as in an untimed step)
        kinds, layers = {}, {}
        for _ in range(a.iters):
            net.timers = []
            net.train_step(x, t)
            torch.cuda.synchronize()
            for kind, name, fl, e0, e1 in net.timers:
                ms = e0.elapsed_time(e1)
                k = kinds.setdefault(kind, [0.0, 0.0])
                k[0] += fl
                k[1] += ms
                l = layers.setdefault(f"{kind}:{name}", [0.0, 0.0])
                l[0] += fl
                l[1] += ms
        net.timers = None
        out["conv_tflops"] = {k: v[0] / v[1] / 1e9 for k, v in kinds.items()}
        out["conv_ms_per_step"] = {k: v[1] / a.iters for k, v in kinds.items()}
        out["conv_layer_tflops"] = {k: round(v[0] / v[1] / 1e9, 1) for k, v in layers.items()}
    out["device_status"] = int(net.L.otf_unet_status())
    print(json.dumps(out))


if __name__ == "__main__":
    _bench()
