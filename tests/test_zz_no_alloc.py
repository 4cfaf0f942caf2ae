"""otf_misfit_noalloc: the misfit entry point for callers that cannot
allocate device memory (their GPU memory is reserved by another allocator,
or they cannot afford cudaMalloc's device synchronisation). It uses the
16 MiB scratch array built into the library instead of caller scratch.

Checked through the C ABI against otf_misfit (caller-provided scratch) on
three calls in a row with different inputs -- the last smaller than the one
before, with another trace length -- so no call can pass on what an earlier
one left in the shared array; and an oversize request must be
refused with an error before anything is launched. This file is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the tolerance the misfit tests use for the device kernels
RTOL = 1e-5


def _traces(seed, n, T):
    rng = np.random.default_rng(seed)
    t = np.arange(T)
    obs = np.stack([np.exp(-((t - rng.uniform(0.2 * T, 0.8 * T)) / (0.02 * T)) ** 2) * np.cos(0.12 * t)
                    for _ in range(n)]).astype(np.float32)
    sim = (np.roll(obs, rng.integers(2, 9), axis=1) + rng.normal(0, 1e-3, obs.shape)).astype(np.float32)
    return sim, obs


def _call(lib, fn_name, kind, sim, obs, torch):
    from otfwi_b200.batch import _declare
    L = _declare(lib)
    n, T = sim.shape
    s = torch.as_tensor(sim).cuda()
    o = torch.as_tensor(obs).cuda()
    adj = torch.full_like(s, float("nan"))
    mis = torch.full((n,), float("nan"), dtype=torch.float64, device=s.device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptrs = [ctypes.c_void_p(x.data_ptr()) for x in (s, o, adj, mis)]
    if fn_name == "otf_misfit":
        nb = int(L.otf_misfit_scratch_bytes(kind, n, T))
        scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=s.device)
        rc = L.otf_misfit(kind, *ptrs, n, T, ctypes.c_void_p(scratch.data_ptr()), nb, st)
    else:
        f = L.otf_misfit_noalloc
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        rc = f(kind, *ptrs, n, T, st)
    torch.cuda.synchronize()
    return rc, mis.cpu().numpy(), adj.cpu().numpy()


# L2, wasserstein, softplus wasserstein, wasserstein_quad, wasserstein_pm (its
# scratch layout differs: 5T float-float values per trace); quad_envelope is
# refused by the entry point
@pytest.mark.parametrize("kind", [1, 2, 0, 3, 5])
def test_noalloc_misfit_matches_allocating_entry_point_twice(lib, kind):
    torch = pytest.importorskip("torch")
    # the third call is smaller than the second and uses another T: it runs
    # over scratch that the larger call left behind
    for call, (seed, n, T) in enumerate([(11, 24, 1500), (12, 40, 4000), (14, 7, 977)]):
        sim, obs = _traces(seed, n, T)
        rc0, m0, a0 = _call(lib, "otf_misfit", kind, sim, obs, torch)
        rc1, m1, a1 = _call(lib, "otf_misfit_noalloc", kind, sim, obs, torch)
        assert rc0 == 0 and rc1 == 0, (call, lib.otf_last_error())
        assert np.all(np.isfinite(a1)) and np.all(np.isfinite(m1))
        np.testing.assert_allclose(m1, m0, rtol=RTOL, atol=0)
        assert np.abs(a1 - a0).max() <= RTOL * max(np.abs(a0).max(), 1e-30), call


def test_noalloc_misfit_rejects_oversize(lib):
    torch = pytest.importorskip("torch")
    sim, obs = _traces(13, 200, 4000)  # 200 traces x 4000 samples: more than the 16 MiB scratch
    lib.otf_clear_error()
    rc, _, adj = _call(lib, "otf_misfit_noalloc", 1, sim, obs, torch)
    assert rc != 0
    assert b"16 MiB" in lib.otf_last_error()
    assert np.all(np.isnan(adj))  # nothing was launched
    lib.otf_clear_error()
