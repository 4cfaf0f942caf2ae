"""GPU tests of the uneven multi-instance group: independent inversions of
different grid sizes, shot counts and T computed as parallel branches of one
CUDA graph (or as chains of branches, otf_multi_set_chains) must give
exactly their stand-alone gradients, and each small
instance's gradient is checked against the FP64 oracle (relative L2 <= 1e-3,
fast numerics)."""
import numpy as np
import pytest

import misfit_oracle as mo
import pml_oracle as po

pytestmark = pytest.mark.gpu

SIZES = [(96, 80, 300, 3), (128, 96, 420, 2), (168, 120, 250, 4)]


def _instances(precision=1):
    from otfwi_b200 import scenarios
    from otfwi_b200.batch import ShotBatch
    out = []
    for i, (X, Z, T, ns) in enumerate(SIZES):
        sc = scenarios.small(X=X, Z=Z, T=T, n_src=ns, n_rec=6, seed=30 + i, f0=0.05)
        b = ShotBatch(X, Z, T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4, precision=precision)
        b.set_model(sc.c_true)
        obs = b.forward()
        b.set_observed(obs)
        b.set_model(sc.c_start)
        out.append((sc, b, obs))
    return out


def test_multi_instance_graph_equals_standalone(lib):
    from otfwi_b200.batch import MultiBatch
    inst = _instances()
    alone = [b.gradient("wasserstein") for _, b, _ in inst]
    m = MultiBatch([b for _, b, _ in inst])
    together = m.gradient("wasserstein")
    for (g0, m0), (g1, m1) in zip(alone, together):
        assert np.array_equal(g0, g1)
        assert m0 == m1
    # a second launch of the same graph reproduces it
    again = m.gradient("wasserstein")
    for (g0, _), (g1, _) in zip(together, again):
        assert np.array_equal(g0, g1)
    # the instances as chains (one at a time, then two at once): the same
    import ctypes
    L = m._lib
    L.otf_multi_set_chains.restype = ctypes.c_int
    L.otf_multi_set_chains.argtypes = [ctypes.c_void_p, ctypes.c_int]
    for chains in (1, 2):
        assert L.otf_multi_set_chains(m._h, chains) == 0
        chained = m.gradient("wasserstein")
        for (g0, m0), (g1, m1) in zip(alone, chained):
            assert np.array_equal(g0, g1) and m0 == m1, chains


def test_multi_instance_gradients_vs_fp64_oracle(lib):
    from otfwi_b200.batch import MultiBatch
    from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask
    inst = _instances()
    res = MultiBatch([b for _, b, _ in inst]).gradient("l2")
    for (sc, b, obs), (g, mis) in zip(inst, res):
        dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML)
        sx, sz = sc.src_xz()
        mx, mz = sc.rec_xz()
        rz, rx = np.where(ring_mask(sc.X, sc.Z, sc.PML, np.where(sc.src_mask), 4))
        acc = np.zeros((sc.Z, sc.X))
        for s in range(sc.n_src):
            gs, _, _ = po.grad(sc.c_start ** 2, np.ones(3), dxp, dzp, sx, sz, sc.source, mx, mz, rx, rz,
                               lambda sim, o=obs[s]: mo.L2(sim, o), s, "f64")
            acc += gs
        ref = acc / sc.n_src
        rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
        print(sc.X, sc.Z, sc.T, sc.n_src, "rel L2 vs FP64 oracle", rel)
        assert rel <= 1e-3
