"""The U-Net's 3x3 convolution and its weight gradient on the tcgen05 tensor
cores (k_conv3x3_umma, k_conv3x3_wgrad_umma: the default paths of
otf_unet_conv3x3 / otf_unet_conv3x3_wgrad) against the numpy oracle (FP64
sums of the same BF16 operands) and against the warp-level mma.sync kernels
they replaced (the small layers through the persistent kernel with resident
weights), over the shapes the network uses and edge shapes: every
output channel count of the network (32, 64, 128, 256), 96, and 512 (two
blocks of 256 channels), grids that are not multiples of the 8 x 16 pixel
tile, the upsampled second input, bias + ReLU and split masked outputs (the
input gradient's form). Convolution outputs are BF16: relative L2 <= 1e-2
against the oracle, as the other U-Net tests; the two kernels sum the same
products in different orders, so they agree to a few BF16 roundings
(relative L2 <= 5e-3). Weight gradients are FP32 sums: relative L2 <= 1e-4.
With the weights packed for bulk copies (otf_unet_conv3x3_packed) the
result is bit-identical. The kernels' bounded waits must all have completed
(device status 0)."""
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


CASES = [
    # N, H, W, c0, c1, up1, cout, split, mask0, relu
    (2, 32, 48, 16, 0, 0, 32, 32, False, 1),
    (1, 20, 36, 32, 0, 0, 64, 64, False, 1),      # H, W not multiples of the tile
    (2, 24, 40, 32, 64, 1, 64, 32, True, 1),      # concat + upsample, split masked output
    (1, 16, 24, 64, 128, 1, 128, 128, False, 1),
    (1, 16, 16, 128, 0, 0, 256, 256, False, 0),
    (1, 8, 16, 256, 0, 0, 512, 256, False, 1),    # two 256-channel blocks
    (3, 9, 11, 48, 0, 0, 96, 96, False, 1),       # ragged tiles, cout 96
    # small layers (persistent kernel, weights resident in shared memory)
    (2, 24, 40, 32, 32, 1, 32, 32, False, 1),     # concat + upsample
    (1, 20, 36, 32, 0, 0, 64, 32, True, 0),       # split masked output, no ReLU
    (5, 40, 24, 16, 0, 0, 32, 32, False, 1),      # ragged last tile row (40 = 32 + 8)
    (1, 16, 16, 32, 0, 0, 192, 64, True, 0),      # few tiles: 192 channels split into 96-channel blocks,
                                                  # the split inside the first block (input-gradient form)
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[1]}x{c[2]}_c{c[3]}+{c[4]}_o{c[6]}" for c in CASES])
def test_umma_conv_vs_oracle_and_legacy(lib, case):
    import torch
    from otfwi_b200.unet import _declare, _p
    N, H, W, c0, c1, up1, cout, split, use_mask, relu = case
    L = _declare(lib)
    rng = np.random.default_rng(sum(case[:7]))
    x0 = rng.standard_normal((N, H, W, c0))
    x1 = rng.standard_normal((N, H // 2, W // 2, c1)) if up1 else (
        rng.standard_normal((N, H, W, c1)) if c1 else None)
    w = rng.standard_normal((9, cout, c0 + c1)) * (1.0 / np.sqrt(9 * (c0 + c1)))
    b = rng.standard_normal(cout).astype(np.float32)
    m0 = np.maximum(rng.standard_normal((N, H, W, split)), 0) if use_mask else None
    X0, Wt = _bf(x0), _bf(w.reshape(-1))
    X1 = _bf(x1) if x1 is not None else None
    M0 = _bf(m0) if m0 is not None else None
    B = torch.as_tensor(b).cuda()
    st = torch.cuda.current_stream().cuda_stream
    outs = {}
    for umma in (1, 0):
        L.otf_unet_set_umma(umma)
        D0 = torch.full((N, H, W, split), float("nan"), dtype=torch.bfloat16, device="cuda")
        D1 = torch.full((N, H, W, max(cout - split, 1)), float("nan"), dtype=torch.bfloat16, device="cuda")
        rc = L.otf_unet_conv3x3(_p(X0), c0, _p(X1), c1, up1, _p(Wt), _p(B), relu, _p(D0), _p(M0),
                                _p(D1) if split < cout else None, None, split, cout, N, H, W, st)
        assert rc == 0, lib.otf_last_error()
        torch.cuda.synchronize()
        outs[umma] = (_np(D0), _np(D1)[..., :cout - split])
    L.otf_unet_set_umma(1)
    # the same convolution with the weights packed for bulk copies: the same
    # shared-memory layout, so the same result bit for bit
    Wp = torch.empty_like(Wt)
    assert L.otf_unet_pack_weights_tc(_p(Wt), cout, c0 + c1, _p(Wp), st) == 0
    P0 = torch.full((N, H, W, split), float("nan"), dtype=torch.bfloat16, device="cuda")
    P1 = torch.full((N, H, W, max(cout - split, 1)), float("nan"), dtype=torch.bfloat16, device="cuda")
    assert L.otf_unet_conv3x3_packed(_p(X0), c0, _p(X1), c1, up1, _p(Wt), _p(Wp), _p(B), relu, _p(P0), _p(M0),
                                     _p(P1) if split < cout else None, None, split, cout, N, H, W, st) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_np(P0), outs[1][0]) and np.array_equal(_np(P1)[..., :cout - split], outs[1][1])
    assert L.otf_unet_status() == 0
    net = uo.Net(np.zeros(uo.n_params(4), np.float32), 4)
    xin = _np(X0)
    if c1:
        xs = _np(X1)
        xin = np.concatenate([xin, net.up(xs) if up1 else xs], axis=-1)
    ref = net.conv(xin, _np(Wt).reshape(9, cout, c0 + c1)) + b
    if relu:
        ref = np.maximum(ref, 0)
    r0 = ref[..., :split] * ((m0 > 0) if use_mask else 1.0)
    r1 = ref[..., split:]
    for umma in (1, 0):
        d0, d1 = outs[umma]
        assert np.all(np.isfinite(d0)) and np.all(np.isfinite(d1)), umma
        e0 = _rel(d0, r0)
        e1 = _rel(d1, r1) if split < cout else 0.0
        print("umma" if umma else "legacy", case, f"rel L2 {e0:.2e} {e1:.2e}")
        assert e0 <= 1e-2 and e1 <= 1e-2
    assert _rel(outs[1][0], outs[0][0]) <= 5e-3
    if split < cout:
        assert _rel(outs[1][1], outs[0][1]) <= 5e-3


def test_umma_conv_persistent_many_tiles(lib):
    """A full-size first layer (16 x 256^2, 32 -> 32 channels): 4096 tiles,
    so each persistent CTA walks several tiles through both accumulator
    buffers; against the mma.sync kernel (relative L2 <= 5e-3)."""
    import torch
    from otfwi_b200.unet import _declare, _p
    L = _declare(lib)
    N, H, W, c, cout = 16, 256, 256, 32, 32
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    X = torch.randn(N, H, W, c, device="cuda", generator=g).to(torch.bfloat16)
    Wt = (torch.randn(9 * cout * c, device="cuda", generator=g) / 17.0).to(torch.bfloat16)
    B = torch.randn(cout, device="cuda", generator=g)
    st = torch.cuda.current_stream().cuda_stream
    outs = {}
    for umma in (1, 0):
        L.otf_unet_set_umma(umma)
        D = torch.full((N, H, W, cout), float("nan"), dtype=torch.bfloat16, device="cuda")
        assert L.otf_unet_conv3x3(_p(X), c, None, 0, 0, _p(Wt), _p(B), 1, _p(D), None, None, None, cout, cout,
                                  N, H, W, st) == 0, lib.otf_last_error()
        torch.cuda.synchronize()
        outs[umma] = D.float()
    L.otf_unet_set_umma(1)
    assert L.otf_unet_status() == 0
    assert torch.isfinite(outs[1]).all()
    e = float(torch.linalg.vector_norm(outs[1] - outs[0]) / torch.linalg.vector_norm(outs[0]))
    print(f"persistent 16x256^2 32->32: rel L2 vs mma.sync {e:.2e}")
    assert e <= 5e-3


WG_CASES = [
    # N, H, W, c0, c1, up1, cout
    (2, 32, 40, 16, 0, 0, 32),      # 16 input channels (16-channel blocks)
    (1, 20, 36, 32, 0, 0, 32),      # ragged tiles, 32 x 32
    (2, 24, 40, 32, 64, 1, 64),     # concat + upsampled second input
    (1, 16, 16, 128, 0, 0, 256),    # two 128-channel output blocks
]


@pytest.mark.parametrize("case", WG_CASES, ids=[f"{c[1]}x{c[2]}_c{c[3]}+{c[4]}_o{c[6]}" for c in WG_CASES])
def test_umma_wgrad_vs_oracle_and_legacy(lib, case):
    import torch
    from otfwi_b200.unet import _declare, _p
    N, H, W, c0, c1, up1, cout = case
    L = _declare(lib)
    rng = np.random.default_rng(7 + sum(case))
    x0 = rng.standard_normal((N, H, W, c0))
    x1 = rng.standard_normal((N, H // 2, W // 2, c1)) if c1 else None
    dz = rng.standard_normal((N, H, W, cout))
    X0, DZ = _bf(x0), _bf(dz)
    X1 = _bf(x1) if x1 is not None else None
    cin = c0 + c1
    sm = torch.cuda.get_device_properties(0).multi_processor_count
    st = torch.cuda.current_stream().cuda_stream
    res = {}
    for umma in (1, 0):
        L.otf_unet_set_umma(2 if umma else 0)  # 2: tcgen05 whatever the layer size
        dW = torch.zeros(9 * cout * cin, dtype=torch.float32, device="cuda")
        assert L.otf_unet_conv3x3_wgrad(_p(X0), c0, _p(X1), c1, up1, _p(DZ), cout, _p(dW), N, H, W, sm, st) == 0
        torch.cuda.synchronize()
        res[umma] = dW.cpu().numpy().reshape(9, cout, cin)
    L.otf_unet_set_umma(1)
    assert L.otf_unet_status() == 0
    net = uo.Net(np.zeros(uo.n_params(4), np.float32), 4)
    xin = _np(X0)
    if c1:
        xin = np.concatenate([xin, net.up(_np(X1))], axis=-1)
    ref = net._wgrad(xin, _np(DZ))
    for umma in (1, 0):
        e = _rel(res[umma], ref)
        print("umma" if umma else "legacy", case, f"wgrad rel L2 {e:.2e}")
        assert e <= 1e-4
