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
