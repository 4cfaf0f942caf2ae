"""GPU tests of the paired step kernels (variant 5: both half-steps of a time
step in one launch, P and A work items handed out by a ticket counter) and of
the launch ordering the fast numerics rely on.

* Variant 5 runs the same device functions as the unfused kernels (variant
  4): traces, gradients, misfits and illumination must be bit-identical, on
  grids whose width is not a multiple of the 128-column block, on points
  inside the damped strips, for every admissible issue lead (the fewest P
  items ahead of the first A item, a middle value and all of them) and
  through the drop-in ABI.
* With and without programmatic dependent launch (OTFWI_PDL=1 / 0, read once
  per process, so each runs in a child process) the default fast gradient is
  identical, and within the fast-numerics tolerance of the CPU oracle.
* The device-side fault reporting of the paired synchronisation (a bounded
  wait that runs out, a ticket count that does not match) reaches the host
  as an error status, without any GPU fault.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

pytestmark = pytest.mark.gpu


def _batch_run(sc, kernel, lead=None, shots=None, misfit="l2"):
    from otfwi_b200.batch import ShotBatch
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4,
                  precision=1, kernel=kernel, shots=shots)
    try:
        if lead is not None:
            b.set_paired_lead(lead)
        b.set_model(sc.c_true)
        obs = b.forward().copy()
        b.set_observed(obs)
        b.set_model(sc.c_start)
        sim = b.forward().copy()
        g, m = b.gradient(misfit)
        illum = b.illumination(5).copy()
        return obs, sim, g.copy(), m, illum
    finally:
        b.close()


def _fmc_small(X=300, Z=136, T=260, n=24, seed=4):
    from otfwi_b200 import scenarios
    return scenarios.fmc(X=X, Z=Z, T=T, n_elem=n, pitch=9, x_first=40, seed=seed)


def test_paired_bit_identical_to_unfused_batched(lib):
    """24-shot FMC gradient on a 300 x 136 grid (width not a multiple of 128):
    every output of variant 5, with the smallest, a middle and the largest
    lead, equals variant 4's bit for bit. (L2 misfit: in 260 steps the far
    receivers of this array record nothing, and the Wasserstein misfits of an
    all-zero observed trace are 0/0, as in the reference.)"""
    sc = _fmc_small()
    ref = _batch_run(sc, 4)
    ncb = -(-sc.X // 128)
    np_items = ncb * -(-sc.Z // 8) * sc.n_src
    for lead in (2 * ncb, 97, np_items, 0):
        out = _batch_run(sc, 5, lead=lead)
        for name, a, b in zip(("obs", "sim", "grad", "misfit", "illum"), out, ref):
            assert np.array_equal(np.asarray(a), np.asarray(b)), (lead, name)


def test_paired_bit_identical_to_unfused_dropin(lib):
    """Through the drop-in ABI (one shot per call, the reference wrapper's
    sequence): the strip case (points inside the damped strips) and a
    101 x 77 grid."""
    from test_dropin_gpu import _keys, _run, _strip_case
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    sc = scenarios.small(X=101, Z=77, T=220, n_src=2, n_rec=7, seed=3, f0=0.05)
    odd = make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
    for name, inp in (("strip", _strip_case()), ("101x77", odd)):
        a = _run(lib, inp, precision=1, kernel=5)
        b = _run(lib, inp, precision=1, kernel=4)
        for k in _keys(b):
            assert np.array_equal(a[k], b[k]), (name, k)


_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/oracle")
import pml_oracle as po, misfit_oracle as mo
from otfwi_b200 import scenarios
from otfwi_b200.batch import ShotBatch
from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask
sc = scenarios.small(X=160, Z=104, T=300, n_src=3, n_rec=8, seed=17, f0=0.04)
b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4, precision=1,
              kernel=int(sys.argv[3]))
b.set_model(sc.c_true); obs = b.forward().copy(); b.set_observed(obs); b.set_model(sc.c_start)
g, m = b.gradient("l2"); b.close()
dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML); sx, sz = sc.src_xz(); mx, mz = sc.rec_xz()
rz, rx = np.where(ring_mask(sc.X, sc.Z, sc.PML, np.where(sc.src_mask), 4))
acc = np.zeros((sc.Z, sc.X))
for s in range(sc.n_src):
    gs, _, _ = po.grad(sc.c_start ** 2, np.ones(3), dxp, dzp, sx, sz, sc.source, mx, mz, rx, rz,
                       lambda v, o=obs[s]: mo.L2(v, o), idx_source=s, mode="f64")
    acc += gs
ref = acc / sc.n_src
err = float(np.linalg.norm(g - ref) / np.linalg.norm(ref))
np.save(sys.argv[2], g)
print(json.dumps({"err": err, "misfit": m}))
"""


def test_fast_gradient_same_with_and_without_pdl(lib, tmp_path):
    """The default fast gradient (unfused kernels, launched with programmatic
    dependent launch unless OTFWI_PDL=0) in two fresh processes: identical
    gradients, each within 1e-3 (relative L2) of the FP64 oracle; and the
    same for the paired kernels."""
    for kernel in ("-1", "5"):
        out = {}
        for pdl in ("1", "0"):
            env = dict(os.environ, OTFWI_PDL=pdl)
            path = str(tmp_path / f"g{pdl}_{kernel}.npy")
            r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, path, kernel], env=env, capture_output=True,
                               text=True, timeout=600)
            assert r.returncode == 0, r.stderr[-2000:]
            res = json.loads(r.stdout.strip().splitlines()[-1])
            assert res["err"] < 1e-3, (kernel, pdl, res)
            out[pdl] = np.load(path)
        assert np.array_equal(out["0"], out["1"]), kernel


def test_paired_fault_reporting(lib):
    """A dependency wait that nothing satisfies gives up after its bound, and
    a paired ticket count and an unfused launch count that do not match are
    flagged: all three reach the host as error bits, and the device keeps
    running work afterwards."""
    import ctypes
    from otfwi_b200 import _lib
    f = lib.otf_selftest_paired_faults
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(ctypes.c_int)]
    bits = ctypes.c_int(0)
    rc = f(ctypes.byref(bits))
    assert rc == 0, (bits.value, lib.otf_last_error())
    assert bits.value & 2 and bits.value & 4 and bits.value & 8
    sc = _fmc_small(X=160, Z=96, T=120, n=4)
    out = _batch_run(sc, 5)
    assert np.abs(out[2]).max() > 0
    _lib.check(lib)
