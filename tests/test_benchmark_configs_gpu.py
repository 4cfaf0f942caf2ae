"""Parity at the benchmark's own configurations, against the FP64 oracle.

* Plain single shot at full size (256 x 256, T = 1500, one source, 32
  receivers, L2 misfit): the faithful drop-in path is bit-identical to the
  reference library (tests/golden/sim_c1.npz, produced by the reference's own
  library on a GPU) -- covered with the other golden cases in
  tests/test_dropin_gpu.py -- and here both numerics are compared with the
  FP64 oracle (oracle/pml_oracle.c, the same algorithm in FP64): traces
  within 1e-5, gradient within 1e-4.
* Full-matrix capture at full size (512 x 512, T = 4000, the 64-element array,
  softplus-normalised Wasserstein): the default fast path (the batched
  engine as the benchmark runs it) on two of the 64 shots -- the first and the
  last element -- against the FP64 oracle's traces and gradient of the same
  shots with the same observed data (max relative trace error <= 1e-5,
  gradient relative L2 <= 1e-4).

Error measures as everywhere in the tests: traces -- max over receivers of
max_{t>=1}|d| / max_t|ref|; gradients -- relative L2 over the grid.
"""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from test_oracle import oracle_case, rel_l2, rel_trace_err  # noqa: E402

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5
GRAD_TOL = 1e-4


def _c1():
    path = os.path.join(GOLDEN, "sim_c1.npz")
    if not os.path.exists(path):
        pytest.skip("sim_c1.npz not generated")
    return dict(np.load(path))


@pytest.fixture(scope="module")
def c1_oracle64():
    d = _c1()
    return d, oracle_case(d, "f64", shots=[0])


@pytest.mark.parametrize("precision", [0, 1])
def test_c1_full_size_vs_fp64_oracle(lib, c1_oracle64, precision):
    from test_dropin_gpu import _run
    d, o64 = c1_oracle64
    res = _run(lib, d, precision=precision, kernel=1)
    et = rel_trace_err(res["traces_all"], o64["traces_all"])
    eg = rel_l2(res["grad_s0"], o64["grad_s0"])
    print(f"C1 {'fast' if precision else 'faithful'}: trace {et:.2e} gradient {eg:.2e}")
    assert et <= TRACE_TOL
    assert eg <= GRAD_TOL
    if precision == 0:
        # the reference library itself, on the same scale
        assert rel_trace_err(d["traces_all"], o64["traces_all"]) <= TRACE_TOL


def _c2_shots():
    return [0, 63]


@pytest.fixture(scope="module")
def c2_case():
    """The benchmark's FMC scenario, the GPU's fast forward of the true model
    as observed data, and the FP64 oracle's traces and gradient (start model)
    of two shots against those observed data."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import misfit_oracle as mo
    import pml_oracle as po
    from otfwi_b200 import scenarios
    from otfwi_b200.batch import ShotBatch
    from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask
    sc = scenarios.fmc()
    shots = _c2_shots()
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4,
                  precision=1, shots=(np.arange(len(shots) + 1), np.asarray(shots)))
    b.set_model(sc.c_true)
    obs = b.forward().copy()
    b.set_observed(obs)
    b.set_model(sc.c_start)
    sim = b.forward().copy()
    g, mis = b.gradient("wasserstein_softplus")
    b.close()
    dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML)
    sx, sz = sc.src_xz()
    mx, mz = sc.rec_xz()
    rz, rx = np.where(ring_mask(sc.X, sc.Z, sc.PML, np.where(sc.src_mask), 4))
    g64 = np.zeros((sc.Z, sc.X))
    sims64 = []
    for i, s in enumerate(shots):
        gs, rec, _ = po.grad(sc.c_start ** 2, np.ones(3), dxp, dzp, sx, sz, sc.source, mx, mz, rx, rz,
                             lambda v, o=obs[i]: mo.wasserstein_softplus(v, o), idx_source=s, mode="f64")
        g64 += gs
        sims64.append(rec)
    return sim, g.copy(), np.stack(sims64), g64 / len(shots)


def test_c2_fast_path_full_size_vs_fp64_oracle(lib, c2_case):
    sim, g, sim64, g64 = c2_case
    et = max(rel_trace_err(sim[i], sim64[i]) for i in range(len(sim)))
    eg = rel_l2(g, g64)
    print(f"C2 fast path, shots {_c2_shots()}: trace {et:.2e} gradient {eg:.2e}")
    assert np.abs(g64).max() > 0
    assert et <= TRACE_TOL
    assert eg <= GRAD_TOL
