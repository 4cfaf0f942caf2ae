"""GPU test of the uneven multi-instance configuration: the four smallest of
the 48 seeded instances (otfwi_b200.uneven.instance_specs), computed as
parallel branches of one CUDA graph, against the FP64 oracle on two shots of
each -- the first and the last element of the instance's array -- (relative
L2 of the shot-mean gradient <= 1e-3, fast numerics)."""
import numpy as np
import pytest

import misfit_oracle as mo
import pml_oracle as po

pytestmark = pytest.mark.gpu


def test_smallest_uneven_instances_vs_fp64_oracle(lib):
    from otfwi_b200.batch import MultiBatch, ShotBatch
    from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask
    from otfwi_b200.uneven import instance_specs, scenario
    specs = instance_specs(48)
    cells = [s["X"] * s["Z"] * s["T"] for s in specs]
    small = sorted(range(len(specs)), key=lambda i: cells[i])[:4]
    n_shots = 2
    batches, scs, obs_all, fired = [], [], [], []
    for i in small:
        sc = scenario(specs[i])
        srcs = np.array([0, sc.n_src - 1], dtype=np.int32)
        shots = (np.arange(n_shots + 1, dtype=np.int32), srcs)
        b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, shots=shots, precision=1)
        b.set_model(sc.c_true)
        obs = b.forward()
        b.set_observed(obs)
        b.set_model(sc.c_start)
        batches.append(b)
        scs.append(sc)
        obs_all.append(obs)
        fired.append(srcs)
    res = MultiBatch(batches).gradient("l2")
    for sc, obs, srcs, (g, _) in zip(scs, obs_all, fired, res):
        dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML)
        sx, sz = sc.src_xz()
        mx, mz = sc.rec_xz()
        rz, rx = np.where(ring_mask(sc.X, sc.Z, sc.PML, np.where(sc.src_mask), 4))
        acc = np.zeros((sc.Z, sc.X))
        for s in range(n_shots):
            gs, _, _ = po.grad(sc.c_start ** 2, np.ones(3), dxp, dzp, sx, sz, sc.source, mx, mz, rx, rz,
                               lambda sim, o=obs[s]: mo.L2(sim, o), int(srcs[s]), "f64")
            acc += gs
        ref = acc / n_shots
        rel = float(np.linalg.norm(g - ref) / np.linalg.norm(ref))
        print(sc.X, sc.Z, sc.T, "rel L2 vs FP64 oracle", rel)
        assert rel <= 1e-3
