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


class SplitSystem:
    """One system spread over the ranks (the config-3 case on several GPUs).

    Every rank holds a share of the particles (32-byte device records, any
    sizes).  A step all-gathers the records (the one exchange the path has:
    32 bytes per particle over NVLink), builds the whole tree on every rank
    and walks only the rank's own particles, so results stay where their
    particles are and need no second collective.  Reloading the particles
    resets a context's OldAcc, so the class keeps its own: |a| of its
    particles' last evaluation (P[].OldAcc, gravtree.c:514-522), passed back to
    the next walk, which reads it only for the rank's own particles.

    `tree` is a library context (ggb200.GravityTree) set to this rank's
    stream; `torch` and `dist` are passed in so that the class runs with gloo
    on CPU tensors in tests."""

    RECORD = 32

    def __init__(self, dist, tree, torch, device):
        self.dist, self.tree, self.torch, self.device = dist, tree, torch, device
        self.world = dist.get_world_size() if dist else 1
        self.rank = dist.get_rank() if dist else 0
        self.counts = None
        self.full = None
        self.oldacc = None      # device, one entry per particle of the system

    def gather(self, local_records):
        """All-gather the ranks' records; returns (all records, counts, own offset)."""
        torch = self.torch
        n_local = local_records.numel() // self.RECORD
        if self.dist is None:
            self.counts = [n_local]
            self.full = local_records
            return self.full, self.counts, 0
        cnt = torch.tensor([n_local], dtype=torch.int64, device=self.device)
        allc = torch.zeros(self.world, dtype=torch.int64, device=self.device)
        self.dist.all_gather_into_tensor(allc, cnt)
        counts = [int(x) for x in allc.cpu().tolist()]
        nmax = max(counts)
        pad = torch.zeros(nmax * self.RECORD, dtype=torch.uint8, device=self.device)
        pad[: n_local * self.RECORD] = local_records
        buf = torch.empty(self.world * nmax * self.RECORD, dtype=torch.uint8, device=self.device)
        self.dist.all_gather_into_tensor(buf, pad)
        parts = [buf[r * nmax * self.RECORD:(r * nmax + counts[r]) * self.RECORD] for r in range(self.world)]
        self.full = torch.cat(parts)
        self.counts = counts
        return self.full, counts, sum(counts[: self.rank])

    def step(self, local_records, d_acc, d_pot, err_tol_force_acc=0.0025, err_tol_theta=0.0):
        """One step for this rank's particles: gather, build, walk the own range.
        d_acc (n_local, 3) and d_pot (n_local) receive the rank's results."""
        torch = self.torch
        full, counts, off = self.gather(local_records)
        n_local, n = counts[self.rank], sum(counts)
        have_old = self.oldacc is not None and self.oldacc.numel() == n
        if not have_old:
            self.oldacc = torch.zeros(n, dtype=torch.float64, device=self.device)
        self.tree.load_device(full, [n])
        self.tree.build()
        active = torch.arange(off, off + n_local, dtype=torch.int32, device=self.device)
        self.tree.evaluate_device(d_acc, d_pot, d_active=active, n_active=n_local,
                                  d_old_acc=self.oldacc if have_old else None,
                                  err_tol_force_acc=err_tol_force_acc, err_tol_theta=err_tol_theta)
        self.oldacc[off:off + n_local] = torch.linalg.norm(d_acc, dim=1)
        return off, n_local
