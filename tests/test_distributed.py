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


class _LinearNet:
    """A stand-in with the preconditioner network's training interface
    (params / grads flat tensors, forward, loss_grad, backward, adam, pack,
    _buffers) on the CPU: out = sum_c x[..., c] * params[c]."""

    def __init__(self, cin, seed):
        import torch
        self.params = torch.as_tensor(np.random.default_rng(seed).standard_normal(cin), dtype=torch.float32)
        self.grads = torch.zeros_like(self.params)

    def pack(self):
        pass

    def forward(self, x):
        self.x = x
        self.out = (x * self.params).sum(-1)
        return self.out

    def loss_grad(self, y, w, inv_norm):
        r = self.out - y
        self.dout = 2.0 * w * r * inv_norm
        return ((w * r * r).sum() * inv_norm).reshape(1)

    def _buffers(self, N, H, W):
        return {"dout": self.dout}

    def backward(self, dout):
        self.grads.copy_((dout[..., None] * self.x).sum((0, 1, 2)))
        return self.grads

    def adam(self, lr):
        self.params -= lr * self.grads


def _dp_data():
    import torch
    rng = np.random.default_rng(3)
    X = torch.as_tensor(rng.standard_normal((12, 8, 8, 3)), dtype=torch.float32)
    Y = (X * torch.tensor([0.5, -1.0, 2.0])).sum(-1)
    return X, Y, torch.ones(8, 8)


def _dp_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from otfwi_b200 import learned
    from otfwi_b200.distributed import dp_average_
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = torch.full((3,), float(rank + 1))
        dp_average_(t)
        net = _LinearNet(3, seed=100 + rank)  # different start on each rank: the broadcast aligns them
        X, Y, w = _dp_data()
        losses = learned.train(net, X, Y, w, steps=30, batch=2, lr=0.05, seed=5)
        np.savez(os.path.join(out, f"dp{rank}.npz"), avg=t.numpy(), params=net.params.numpy(),
                 losses=np.array(losses))
    finally:
        dist.destroy_process_group()


def test_data_parallel_training_two_gloo_ranks(tmp_path):
    """The preconditioner's data-parallel training loop (learned.train with a
    process group): gradients averaged by one all-reduce per step, parameters
    identical on every rank after training, the loss history the ranks'
    mean, and the model converging on its synthetic linear target."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_dp_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    d = [np.load(tmp_path / f"dp{r}.npz") for r in range(2)]
    assert np.array_equal(d[0]["avg"], np.full(3, 1.5)) and np.array_equal(d[1]["avg"], np.full(3, 1.5))
    assert np.array_equal(d[0]["params"], d[1]["params"])
    assert np.array_equal(d[0]["losses"], d[1]["losses"])
    assert d[0]["losses"][-1] < 0.05 * d[0]["losses"][0]
    np.testing.assert_allclose(d[0]["params"], [0.5, -1.0, 2.0], atol=0.5)


def _agree_worker(rank, world, port, out):
    import torch.distributed as dist
    from otfwi_b200.distributed import agree_ints
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank's own autotuner result differs (timing noise); rank 0's wins
        got = agree_ints([4 - 2 * rank, 4 + rank])
        np.save(os.path.join(out, f"agree{rank}.npy"), np.array(got))
    finally:
        dist.destroy_process_group()


def test_ranks_agree_on_rank0_tuning(tmp_path):
    """bench.py's multi-rank run: every rank ends with rank 0's (kernel,
    tile), so all GPUs of a scaling run execute the same kernels."""
    import torch.multiprocessing as mp
    from otfwi_b200.distributed import agree_ints
    assert agree_ints([4, 3]) == [4, 3]  # no process group: unchanged
    port = _free_port()
    mp.start_processes(_agree_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        assert np.load(tmp_path / f"agree{r}.npy").tolist() == [4, 4]


def test_training_single_process_unchanged():
    """Without a process group the loop is the single-GPU one: no collective."""
    from otfwi_b200 import learned
    X, Y, w = _dp_data()
    net = _LinearNet(3, seed=1)
    losses = learned.train(net, X, Y, w, steps=10, batch=2, lr=0.05, seed=5)
    assert len(losses) == 10 and losses[-1] < losses[0]
