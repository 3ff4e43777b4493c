"""Multi-GPU plumbing: one process per GPU, independent systems per rank.

The tree-gravity path shards by system: every rank builds and walks its own
systems (its own galaxy in the weak-scaling bench, its share of an ensemble or
of a serving stream), so the data path has no collective.  The process group
(NCCL on GPUs, gloo on CPU in the tests) only carries barriers and the
max-over-ranks timing.  Ranks take the same collective steps in the same order.
"""
import datetime
import os

import numpy as np


def world():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def init(backend="nccl", timeout_s=300):
    """Start the process group when launched with WORLD_SIZE > 1; returns the
    torch.distributed module or None for a single process."""
    size, _, _ = world()
    if size <= 1:
        return None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def rank_seed(base, rank):
    """Seed of rank `rank`'s independent system (rank 0 keeps the base seed)."""
    return int(base) + 7919 * int(rank)


def assign_systems(counts, size, rank):
    """Indices of the systems rank `rank` of `size` evaluates.

    Longest-processing-time greedy on particle counts (a system's cost grows
    with N), deterministic: every rank computes the same partition."""
    counts = np.asarray(counts, dtype=np.int64)
    order = np.argsort(-counts, kind="stable")
    load = np.zeros(size, dtype=np.int64)
    owner = np.empty(counts.size, dtype=np.int64)
    for s in order:
        r = int(np.argmin(load))
        owner[s] = r
        load[r] += counts[s]
    return np.flatnonzero(owner == rank)


def _reduce(dist, value, op, device):
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(dist, value, device="cpu"):
    if dist is None:
        return float(value)
    return _reduce(dist, value, dist.ReduceOp.MAX, device)


def sum_over_ranks(dist, value, device="cpu"):
    if dist is None:
        return float(value)
    return _reduce(dist, value, dist.ReduceOp.SUM, device)
