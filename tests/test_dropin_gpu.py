"""GPU parity of the drop-in C ABI (libotfwi.so) against the reference
library's own outputs (tests/golden/sim_*.npz) and the CPU oracle, through
the reference wrapper's call sequence (tests/abi_driver.py).

Faithful mode (the default) restates the reference's arithmetic operation by
operation, so it is required to be bit-identical to the reference library
and to the f32 oracle: traces (t >= 1) and gradients, every sample.
Against the FP64 oracle, and for the fast (FP32-sum) mode, the error
measures are: traces -- max over receivers of max_{t>=1}|d| / max_t|ref|
(tolerance 1e-5 faithful, 1e-4 fast); gradients -- relative L2 over the grid
(1e-4 faithful, 1e-3 fast).
"""
import glob
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from abi_driver import run_abi  # noqa: E402
from test_oracle import oracle_case, rel_l2, rel_trace_err  # noqa: E402

pytestmark = pytest.mark.gpu


def _cases():
    import make_sim_golden
    return make_sim_golden.cases()


def _run(lib, inp, precision=0, tile=0, kernel=1):
    from otfwi_b200 import _lib
    os.environ["OTFWI_PRECISION"] = str(precision)
    os.environ["OTFWI_TILE"] = str(tile)
    os.environ["OTFWI_KERNEL"] = str(kernel)
    try:
        return run_abi(lib, **inp, check=lambda: _lib.check(lib))
    finally:
        os.environ.pop("OTFWI_PRECISION", None)
        os.environ.pop("OTFWI_TILE", None)
        os.environ.pop("OTFWI_KERNEL", None)


def _keys(ref):
    return [k for k in ref if k.startswith(("traces_", "sim_s", "grad_s"))]


def _assert_identical(res, ref, label):
    for k in _keys(ref):
        a, b = np.asarray(res[k]), np.asarray(ref[k])
        if not k.startswith("grad_s"):
            a, b = a[:, 1:], b[:, 1:]  # column 0 is never simulated
        nd = int(np.sum(a != b))
        assert nd == 0, (label, k, nd, a.size)


def _assert_close(res, ref, ttol, gtol, label):
    errs = {}
    for k in _keys(ref):
        if k.startswith("grad_s"):
            errs[k] = rel_l2(res[k], ref[k])
            assert errs[k] <= gtol, (label, k, errs[k])
        else:
            errs[k] = rel_trace_err(res[k], ref[k])
            assert errs[k] <= ttol, (label, k, errs[k])
    return errs


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "sim_*.npz"))),
                         ids=os.path.basename)
def test_dropin_bit_identical_to_reference_library(lib, path):
    d = dict(np.load(path))
    _assert_identical(_run(lib, d), d, "faithful vs reference library")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "sim_*.npz"))),
                         ids=os.path.basename)
def test_fast_mode_close_to_reference_library(lib, path):
    d = dict(np.load(path))
    errs = _assert_close(_run(lib, d, precision=1), d, 1e-4, 1e-3, "fast vs reference library")
    print(os.path.basename(path), {k: f"{v:.2e}" for k, v in errs.items()})


@pytest.mark.parametrize("name", ["small", "medium", "general"])
def test_dropin_matches_oracles(lib, name):
    inp = _cases()[name]
    res = _run(lib, inp)
    _assert_identical(res, oracle_case(inp, "f32"), "faithful vs oracle f32")
    _assert_close(res, oracle_case(inp, "f64"), 1e-5, 1e-4, "faithful vs oracle f64")


@pytest.mark.parametrize("tile", [1, 2, 3, 4])
def test_tile_shapes_bit_identical(lib, tile):
    inp = _cases()["medium"]
    base = _run(lib, inp, tile=0, kernel=0)
    res = _run(lib, inp, tile=tile)
    for k in base:
        assert np.array_equal(base[k], res[k]), (tile, k)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("tile", [0, 1, 4])
def test_persistent_tma_kernels_bit_identical_to_per_tile(lib, tile, precision):
    """The persistent TMA-pipelined step kernels compute with the same device
    code as the one-tile-per-CTA kernels: identical results."""
    inp = _cases()["medium"]
    a = _run(lib, inp, precision=precision, tile=tile, kernel=0)
    b = _run(lib, inp, precision=precision, tile=tile, kernel=1)
    for k in a:
        assert np.array_equal(a[k], b[k]), (tile, precision, k)


def _strip_case():
    """Sources and receivers inside the damped strips (the split component
    Q is injected into and recorded from there)."""
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    sc = scenarios.small(X=112, Z=90, T=260, n_src=2, n_rec=6, seed=9, f0=0.05)
    sc.src_mask[:] = False
    sc.src_mask[10, 30] = True   # inside the top strip
    sc.src_mask[50, 8] = True    # inside the left strip
    sc.rec_mask[:] = False
    sc.rec_mask[12, [20, 50, 80]] = True
    sc.rec_mask[[40, 60], 104] = True
    sc.rec_mask[86, 60] = True   # within 4 cells of the edge: records zeros
    return make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))


@pytest.mark.parametrize("tile", [0, 1, 4])
def test_strip_split_kernels_close_to_oracle(lib, tile):
    """Fast numerics with P everywhere and the split component only on damped
    cells: within the fast-mode tolerance of the FP64 oracle and of the
    split-field fast kernels, on the medium case and on a case with sources
    and receivers inside the strips."""
    for inp in (_cases()["medium"], _strip_case()):
        res = _run(lib, inp, precision=1, tile=tile, kernel=2)
        _assert_close(res, oracle_case(inp, "f64"), 1e-4, 1e-3, f"split vs oracle f64 tile {tile}")
        ref = _run(lib, inp, precision=1, tile=tile, kernel=1)
        _assert_close(res, ref, 1e-4, 1e-3, f"split vs split-field fast tile {tile}")


@pytest.mark.parametrize("rows", [8, 24, 64, 200])
def test_streaming_kernels_close_to_oracle(lib, rows):
    """z-streaming strips (kernel 3) with several segment heights: on the
    medium case and the strip case (points inside the damped strips) within
    the fast-mode tolerance of the FP64 oracle; on these and on a grid wider
    than two strips whose width is not a multiple of the strip, identical to
    the strip-split kernels (with dt = dx the two compute the same operations
    in the same order). On the wide grid some receivers see only numerical
    precursors within T and one shot's gradient is of the order of FP32
    subnormals (its source is out of reach of every receiver), so its oracle
    check is normalised by the largest value of each quantity over all shots."""
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    os.environ["OTFWI_STREAM_ROWS"] = str(rows)
    try:
        sc = scenarios.small(X=268, Z=84, T=220, n_src=2, n_rec=7, seed=12, f0=0.05)
        wide = make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
        for name, inp in (("medium", _cases()["medium"]), ("strip", _strip_case()), ("wide", wide)):
            res = _run(lib, inp, precision=1, kernel=3)
            ref64 = oracle_case(inp, "f64")
            if name == "wide":
                fam = lambda k: k.rstrip("0123456789")
                scale = {}
                for k in _keys(ref64):
                    scale[fam(k)] = max(scale.get(fam(k), 0.0), float(np.abs(ref64[k]).max()))
                for k in _keys(ref64):
                    a, b = np.asarray(res[k], np.float64), np.asarray(ref64[k])
                    assert np.abs(a - b).max() <= 1e-4 * scale[fam(k)], (name, k)
            else:
                _assert_close(res, ref64, 1e-4, 1e-3, f"stream vs oracle f64 {name} rows {rows}")
            ref = _run(lib, inp, precision=1, tile=4, kernel=2)
            _assert_identical(res, ref, f"stream vs strip-split {name} rows {rows}")
    finally:
        os.environ.pop("OTFWI_STREAM_ROWS", None)


def test_unfused_kernels_close_to_oracle(lib):
    """Unfused streaming half-steps (kernel 4): within the fast-mode tolerance
    of the FP64 oracle on the medium case, the strip case and grids whose
    width is not a multiple of the 128-column block or of 4; identical to the
    strip-split kernels (with dt = dx the damped and undamped A updates round
    the same way, so the two compute the same operations)."""
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    cases = [("medium", _cases()["medium"]), ("strip", _strip_case())]
    for X, Z, seed in ((268, 84, 12), (101, 77, 3)):
        sc = scenarios.small(X=X, Z=Z, T=220, n_src=2, n_rec=7, seed=seed, f0=0.05)
        cases.append((f"{X}x{Z}", make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))))
    for name, inp in cases:
        res = _run(lib, inp, precision=1, kernel=4)
        ref64 = oracle_case(inp, "f64")
        fam = lambda k: k.rstrip("0123456789")
        scale = {}
        for k in _keys(ref64):
            scale[fam(k)] = max(scale.get(fam(k), 0.0), float(np.abs(ref64[k]).max()))
        for k in _keys(ref64):
            a, b = np.asarray(res[k], np.float64), np.asarray(ref64[k])
            assert np.abs(a - b).max() <= 1e-4 * scale[fam(k)], (name, k)
        ref = _run(lib, inp, precision=1, tile=4, kernel=2)
        _assert_identical(res, ref, f"unfused vs strip-split {name}")


def test_odd_grid_sizes_every_tile(lib):
    """Grids that are not multiples of any tile shape, both kernel variants."""
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    sc = scenarios.small(X=101, Z=77, T=200, n_src=1, n_rec=5, seed=3)
    inp = make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
    ref = oracle_case(inp, "f32")
    for tile in range(5):
        for kernel in (0, 1):
            _assert_identical(_run(lib, inp, tile=tile, kernel=kernel), ref, f"odd grid tile {tile} k{kernel}")
    ref64 = oracle_case(inp, "f64")
    for tile in (0, 1, 4):
        _assert_close(_run(lib, inp, precision=1, tile=tile, kernel=2), ref64, 1e-4, 1e-3,
                      f"odd grid split tile {tile}")


def test_edge_receiver_records_zero(lib):
    """A receiver on a never-updated cell (within 4 cells of the edge) records
    zeros, as in the reference."""
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    sc = scenarios.small(X=96, Z=64, T=150, n_src=1, n_rec=4, seed=2)
    sc.rec_mask[sc.PML + 6, 2] = True  # x = 2: outside 4 <= x < X-4
    inp = make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
    res = _run(lib, inp)
    assert np.all(res["traces_all"][0] == 0.0)
    assert np.abs(res["traces_all"][1:]).max() > 0


def test_invalid_source_position_is_reported(lib):
    from otfwi_b200 import _lib
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    sc = scenarios.small(X=96, Z=64, T=50, n_src=1, n_rec=4, seed=2)
    sc.src_mask[:] = False
    sc.src_mask[2, 40] = True  # z = 2: a cell the scheme never updates
    inp = make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
    with pytest.raises(_lib.OtfwiError, match="source 0"):
        _run(lib, inp)


def test_hilbert_matches_fft_definition(lib):
    from otfwi_b200._lib import c_float_p
    rng = np.random.default_rng(0)
    for N in (64, 101, 500):
        x = rng.standard_normal(N).astype(np.float32)
        s90 = np.zeros(N, np.float32)
        env = np.zeros(N, np.float32)
        lib.hilbert(x.ctypes.data_as(c_float_p), s90.ctypes.data_as(c_float_p),
                    env.ctypes.data_as(c_float_p), N)
        X = np.fft.fft(x.astype(np.float64))
        X[N // 2: 2 * (N // 2)] = 0
        y = np.fft.ifft(X) * N
        assert np.allclose(s90, 2 * y.imag / N, atol=1e-5)
        assert np.allclose(env, 2 * np.abs(y) / N, atol=1e-5)
