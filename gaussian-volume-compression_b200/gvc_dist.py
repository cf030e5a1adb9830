"""Multi-GPU plumbing of the training step (one process per GPU, torch.distributed).

The path shards by sample points: every rank holds all Gaussians (and rebuilds the
Gaussian LBVH itself: the build is cheap and identical everywhere) and its own sample
set; the forward is independent per sample; the only exchange is one sum all-reduce of
the per-Gaussian gradients ([P, 12] floats) after the backward.
"""
import os

import torch
import torch.distributed as dist


def init_from_env(backend="nccl", timeout_s=120):
    """Initialises the default process group from RANK / WORLD_SIZE / MASTER_* (torchrun)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def shard_range(n, rank, world):
    """Contiguous block [lo, hi) of n items owned by `rank` (sizes differ by at most 1)."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def allreduce_grads(grads):
    """Sums a list of gradient tensors across ranks with ONE all-reduce of a flat buffer."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return grads
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    out, off = [], 0
    for g in grads:
        n = g.numel()
        out.append(flat[off:off + n].view_as(g))
        off += n
    return out


def max_over_ranks(x, device=None):
    """Max of a float across ranks (the timing rule for multi-GPU numbers)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
