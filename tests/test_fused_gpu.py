"""GPU tests of the row-lag fused step kernels (variant 6: a warp computes
P(t) of a row and the A half-step four rows behind it from a register
window, one launch and one pass over the fields per step, no dependency
between CTAs). They run the unfused kernels' cell arithmetic operation for
operation, so every output must be bit-identical to variant 4's: traces,
boundary-ring-based gradients, misfits and illumination, for chunk heights
from the minimum to more than the grid, grids whose width is not a multiple
of the 120-column strip, points inside the damped strips, and through the
drop-in ABI."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

pytestmark = pytest.mark.gpu


def _batch_run(sc, kernel, rows=None, misfit="l2"):
    from otfwi_b200.batch import ShotBatch
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4,
                  precision=1, kernel=kernel)
    try:
        if rows is not None:
            b.set_fused_rows(rows)
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


@pytest.mark.parametrize("rows", [8, 20, 64, 200])
def test_fused_bit_identical_to_unfused_batched(lib, rows):
    """24-shot FMC gradient on a 300 x 136 grid (three 120-column strips, the
    last ragged) with chunks of 8, 20, 64 and 200 rows."""
    from otfwi_b200 import scenarios
    sc = scenarios.fmc(X=300, Z=136, T=260, n_elem=24, pitch=9, x_first=40, seed=4)
    ref = _batch_run(sc, 4)
    out = _batch_run(sc, 6, rows=rows)
    for name, a, b in zip(("obs", "sim", "grad", "misfit", "illum"), out, ref):
        assert np.array_equal(np.asarray(a), np.asarray(b)), (rows, name)


def test_fused_bit_identical_to_unfused_dropin(lib):
    """Through the drop-in ABI: sources and receivers inside the damped
    strips, a 101 x 77 grid and a 268 x 84 grid."""
    from test_dropin_gpu import _keys, _run, _strip_case
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    cases = [("strip", _strip_case())]
    for X, Z, seed in ((101, 77, 3), (268, 84, 12)):
        sc = scenarios.small(X=X, Z=Z, T=220, n_src=2, n_rec=7, seed=seed, f0=0.05)
        cases.append((f"{X}x{Z}", make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))))
    for name, inp in cases:
        a = _run(lib, inp, precision=1, kernel=6)
        b = _run(lib, inp, precision=1, kernel=4)
        for k in _keys(b):
            assert np.array_equal(a[k], b[k]), (name, k)
