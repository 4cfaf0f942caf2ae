"""Multi-rank host logic on CPU: two gloo ranks shard the shots of a small
problem, each computes its shots' gradients with the CPU oracle (the
checker), and one all-reduce must reproduce the single-process shot mean."""
import os
import socket

import numpy as np
import pytest

import misfit_oracle as mo
import pml_oracle as po


def _problem():
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask
    sc = scenarios.small(X=72, Z=64, T=120, n_src=3, n_rec=5, seed=4, f0=0.06)
    dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML)
    sx, sz = sc.src_xz()
    mx, mz = sc.rec_xz()
    rz, rx = np.where(ring_mask(sc.X, sc.Z, sc.PML, np.where(sc.src_mask), 4))
    return sc, dxp, dzp, sx, sz, mx, mz, rx, rz


def _shot_grad(s):
    sc, dxp, dzp, sx, sz, mx, mz, rx, rz = _problem()
    obs = po.simulate(sc.c_true ** 2, np.ones(3), dxp, dzp, sx, sz, sc.source, mx, mz, s, "f32")
    g, _, mis = po.grad(sc.c_start ** 2, np.ones(3), dxp, dzp, sx, sz, sc.source, mx, mz, rx, rz,
                        lambda sim: mo.L2(sim, obs), s, "f32")
    return g, mis


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from otfwi_b200.distributed import distributed_gradient
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, m = distributed_gradient(_shot_grad, 3, rank, world, (64, 72))
        np.savez(os.path.join(out, f"rank{rank}.npz"), g=g, m=m)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_shot_once():
    from otfwi_b200.distributed import shard
    for n in (1, 5, 64):
        for w in (1, 2, 3, 8):
            got = sorted(i for r in range(w) for i in shard(n, w, r))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def test_two_gloo_ranks_match_single_process(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    ref_g = np.zeros((64, 72))
    ref_m = 0.0
    for s in range(3):
        g, m = _shot_grad(s)
        ref_g += g
        ref_m += m
    ref_g /= 3
    for r in range(2):
        d = np.load(tmp_path / f"rank{r}.npz")
        np.testing.assert_allclose(d["g"], ref_g, rtol=1e-12, atol=1e-12 * np.abs(ref_g).max())
        assert abs(float(d["m"]) - ref_m) <= 1e-12 * abs(ref_m)
