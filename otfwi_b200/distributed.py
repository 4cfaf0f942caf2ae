"""Multi-GPU FWI gradient: shots (or whole acquisitions) sharded over ranks,
one reduction per gradient; and the data-parallel step of the
preconditioner's training (each rank its own micro-batch, one all-reduce of
the flat parameter gradient per step).

The reference runs every shot serially on one GPU (cuda_interface_pml.py:
225-236: grad_acc += grad per shot, then / n_source). Shots are
independent, so each rank computes the gradient sum and misfit sum of its own
shots and one all-reduce (NCCL over NVLink between GPUs; gloo on CPU in the
tests) forms the total; the shot mean divides by the global shot count, as
the reference wrapper does. No data-path collective runs inside a time step.
"""
import numpy as np


def shard(n_items, world, rank):
    """Round-robin shard of item indices for one rank."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside world of size {world}")
    return list(range(rank, n_items, world))


def allreduce_sum_(tensors, group=None):
    """In-place sum over ranks of each torch tensor (any backend)."""
    import torch.distributed as dist
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return tensors


def distributed_gradient(shot_gradient, n_shots, rank, world, shape, group=None, device="cpu"):
    """Shot-mean gradient and summed misfit over all ranks.

    shot_gradient(s) -> (grad [shape] array-like, misfit float) computes one
    shot on this rank's device. Returns (grad_mean, misfit_sum) as numpy on
    every rank."""
    import torch
    g = torch.zeros(shape, dtype=torch.float64, device=device)
    m = torch.zeros(1, dtype=torch.float64, device=device)
    for s in shard(n_shots, world, rank):
        gs, ms = shot_gradient(s)
        g += torch.as_tensor(np.asarray(gs), dtype=torch.float64, device=device)
        m += float(ms)
    allreduce_sum_([g, m], group=group)
    return (g / n_shots).cpu().numpy(), float(m.item())


def shard_block(n_items, world, rank):
    """Contiguous balanced block [lo, hi) of item indices for one rank (the
    first n_items % world ranks take one item more)."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside world of size {world}")
    q, r = divmod(n_items, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


class ShardedShots:
    """The shots of ONE acquisition split over the ranks of a process group.

    Replaces the reference's serial per-shot loop (cuda_interface_pml.py:
    225-236: grad_acc += grad per shot, then / n_source; mse likewise): rank r
    owns a contiguous block of the shot table, runs all of its shots in one
    batched gradient (its own GPU, its own CUDA graph), scales its local shot
    mean by n_local / n_total and one all-reduce (NCCL over NVLink between
    GPUs; gloo on CPU) sums the gradient and the misfit over the ranks. Every
    rank ends with the acquisition's shot-mean gradient and total misfit;
    nothing crosses GPUs inside a time step and no gradient visits the host.

    ``make_batch(shots)`` builds a batch object (``ShotBatch`` or anything
    with its set_model / set_observed / forward / gradient / objective /
    illumination methods) for a shot table ``(ptr, srcs)``; ``grid`` is (Z,
    X); ``device`` is where the reduction runs (this rank's CUDA device for
    NCCL, cpu for gloo)."""

    def __init__(self, make_batch, shot_ptr, shot_srcs, grid, group=None, device="cpu"):
        import torch
        self.torch = torch
        self.grid = tuple(int(v) for v in grid)
        self.group = group
        self.device = torch.device(device)
        ptr = np.asarray(shot_ptr, np.int64)
        srcs = np.asarray(shot_srcs, np.int64)
        self.n_total = len(ptr) - 1
        self.world, self.rank = world_of(group)
        self.lo, self.hi = shard_block(self.n_total, self.world, self.rank)
        self.n_local = self.hi - self.lo
        lp = ptr[self.lo:self.hi + 1] - ptr[self.lo]
        ls = srcs[ptr[self.lo]:ptr[self.hi]]
        self.batch = make_batch((lp, ls)) if self.n_local > 0 else None

    @property
    def n_shots(self):
        """Shots of the whole acquisition."""
        return self.n_total

    def close(self):
        if self.batch is not None and hasattr(self.batch, "close"):
            self.batch.close()
        self.batch = None

    def local(self, a):
        """This rank's rows of an array over every shot of the acquisition."""
        return a[self.lo:self.hi]

    def set_model(self, c=None, cquad=None):
        if self.batch is not None:
            self.batch.set_model(c=c, cquad=cquad)

    def set_observed(self, obs_local):
        """Observed traces of this rank's shots [n_local, n_rec, T]."""
        if self.batch is not None:
            self.batch.set_observed(obs_local)

    def forward(self, out=None):
        """Traces of this rank's shots (no collective)."""
        return self.batch.forward(out=out) if self.batch is not None else None

    def _reduce(self, tensors):
        if self.world > 1:
            allreduce_sum_(tensors, group=self.group)
        return tensors

    def gradient(self, misfit="wasserstein", grad=None, misfit_out=None):
        """(shot-mean gradient of the whole acquisition [Z, X], total misfit
        [1] float64) as tensors on this rank's reduction device."""
        torch = self.torch
        dev = self.device
        shape = self.grid
        g = grad
        m = misfit_out
        if self.batch is not None:
            if dev.type == "cuda":
                g = g if g is not None else torch.empty(shape, dtype=torch.float32, device=dev)
                m = m if m is not None else torch.empty(1, dtype=torch.float64, device=dev)
                self.batch.gradient(misfit, grad=g, misfit_out=m)
            else:
                gh, mh = self.batch.gradient(misfit)
                g = torch.as_tensor(np.asarray(gh, np.float32)).to(dev).clone()
                m = torch.tensor([float(mh)], dtype=torch.float64, device=dev)
            g.mul_(self.n_local / self.n_total)
        else:
            g = torch.zeros(shape, dtype=torch.float32, device=dev) if g is None else g.zero_()
            m = torch.zeros(1, dtype=torch.float64, device=dev) if m is None else m.zero_()
        self._reduce([g, m])
        return g, m

    def objective(self, misfit="wasserstein"):
        """Total misfit of every shot of the acquisition (forward only)."""
        torch = self.torch
        v = self.batch.objective(misfit) if self.batch is not None else 0.0
        m = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self._reduce([m])
        return float(m.item())

    def illumination(self, every=8, out=None):
        """Sum over every shot of the acquisition of the forward's P^2."""
        torch = self.torch
        if self.batch is not None:
            if self.device.type == "cuda":
                out = out if out is not None else torch.empty(self.grid, dtype=torch.float32,
                                                              device=self.device)
                self.batch.illumination(every, out=out)
            else:
                out = torch.as_tensor(np.asarray(self.batch.illumination(every), np.float32)).to(self.device)
        else:
            out = torch.zeros(self.grid, dtype=torch.float32, device=self.device) if out is None \
                else out.zero_()
        self._reduce([out])
        return out


def world_of(group=None):
    """(world size, rank) of an initialised process group, else (1, 0)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def dp_average_(grads, group=None):
    """Data-parallel gradient: replace a flat parameter gradient by its mean
    over ranks (one all-reduce; a no-op in a single process). With each
    rank's loss normalised over its own micro-batch, the mean is the gradient
    of the mean loss over the global batch."""
    import torch.distributed as dist
    world, _ = world_of(group)
    if world > 1:
        dist.all_reduce(grads, op=dist.ReduceOp.SUM, group=group)
        grads.div_(world)
    return grads


def broadcast_params_(params, group=None):
    """Rank 0's parameters on every rank (before data-parallel training)."""
    import torch.distributed as dist
    world, _ = world_of(group)
    if world > 1:
        dist.broadcast(params, src=0, group=group)
    return params


def agree_ints(values, group=None, device="cpu"):
    """Rank 0's list of small integers on every rank (one broadcast; the
    values themselves in a single process). Used so that every rank runs the
    kernel variant and tile shape that rank 0's autotuner chose, whatever the
    timing noise of each rank's own tuning."""
    import torch
    import torch.distributed as dist
    world, _ = world_of(group)
    if world == 1:
        return [int(v) for v in values]
    t = torch.tensor([int(v) for v in values], dtype=torch.int64, device=device)
    dist.broadcast(t, src=0, group=group)
    return [int(v) for v in t.cpu().tolist()]
