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
    sizes).  A step all-gathers the records (32 bytes per particle over
    NVLink), builds the whole tree on every rank, and each rank walks one
    contiguous range of the Peano-Hilbert order -- the way the reference cuts
    its space-filling curve into domains of equal work (domain.c:2224-2300) --
    so a walk group's targets are neighbours whatever order the shares came
    in.  The ranges are equal in the number of targets on the first step and
    equal in work after that: the cut points split the cumulative interaction
    count each particle had in the previous step (its cost), taken along the
    new order.  The ranks' results (force, potential, interaction count) are
    then all-gathered, so that every rank has every particle's, and each
    returns its own particles'.  The relative criterion's OldAcc (|a| of every
    particle's last evaluation, P[].OldAcc, gravtree.c:514-522) and the costs
    are kept per particle in gathered load order, and only while the ranks'
    share sizes are the same as in the previous step (otherwise a load index
    would name another particle).

    `tree` is a library context (ggb200.GravityTree) set to this rank's
    stream; `torch` and `dist` are passed in so that the class runs with gloo
    on CPU tensors in tests."""

    RECORD = 32

    def __init__(self, dist, tree, torch, device, balance=True):
        self.dist, self.tree, self.torch, self.device = dist, tree, torch, device
        self.world = dist.get_world_size() if dist else 1
        self.rank = dist.get_rank() if dist else 0
        self.balance = balance
        self.counts = None
        self.full = None
        self.oldacc = None      # one entry per particle of the system, gathered load order
        self.cost = None        # interactions of each particle's last walk, gathered load order
        self.kept_counts = None
        self.last_cuts = None

    def _all_gather_rows(self, rows, sizes):
        """Concatenation over the ranks of each rank's `rows` (sizes[r] rows
        of the same width), with one padded all-gather."""
        torch = self.torch
        if self.dist is None:
            return rows
        width = rows.shape[1]
        nmax = max(sizes)
        # NCCL gathers device memory directly; gloo (CPU tests) only host memory
        where = "cpu" if self.dist.get_backend() == "gloo" else rows.device
        pad = torch.zeros((nmax, width), dtype=rows.dtype, device=where)
        pad[: rows.shape[0]] = rows
        buf = torch.empty((self.world * nmax, width), dtype=rows.dtype, device=where)
        self.dist.all_gather_into_tensor(buf, pad)
        out = torch.cat([buf[r * nmax:r * nmax + sizes[r]] for r in range(self.world)])
        return out.to(rows.device)

    def gather(self, local_records):
        """All-gather the ranks' records; returns (all records, counts, own offset)."""
        torch = self.torch
        n_local = local_records.numel() // self.RECORD
        if self.dist is None:
            self.counts = [n_local]
            self.full = local_records
            return self.full, self.counts, 0
        where = "cpu" if self.dist.get_backend() == "gloo" else self.device
        cnt = torch.tensor([n_local], dtype=torch.int64, device=where)
        allc = torch.zeros(self.world, dtype=torch.int64, device=where)
        self.dist.all_gather_into_tensor(allc, cnt)
        counts = [int(x) for x in allc.cpu().tolist()]
        full = self._all_gather_rows(local_records.view(-1, self.RECORD), counts)
        self.full = full.reshape(-1)
        self.counts = counts
        return self.full, counts, sum(counts[: self.rank])

    def cuts(self, order, n):
        """Sorted positions where each rank's range starts (world + 1 entries):
        equal counts, or equal cumulative cost along `order` when costs are known."""
        torch = self.torch
        W = self.world
        if not self.balance or self.cost is None or W == 1:
            return [r * n // W for r in range(W + 1)]
        cum = torch.cumsum(self.cost[order.long()].double() + 1.0, 0)   # +1: no range without particles' own work
        total = float(cum[-1])
        goals = torch.tensor([total * r / W for r in range(1, W)], dtype=torch.float64, device=cum.device)
        inner = torch.searchsorted(cum, goals).cpu().tolist()
        return [0] + [min(max(int(c), 0), n) for c in inner] + [n]

    def step(self, local_records, d_acc, d_pot, err_tol_force_acc=0.0025, err_tol_theta=0.0):
        """One step for this rank's particles: gather, build, walk the rank's
        Peano-Hilbert range, exchange the results.  d_acc (n_local, 3) and
        d_pot (n_local) receive the results of the rank's own particles."""
        torch = self.torch
        full, counts, off = self.gather(local_records)
        n_local, n = counts[self.rank], sum(counts)
        have_old = self.oldacc is not None and self.kept_counts == counts
        if not have_old:
            self.oldacc = torch.zeros(n, dtype=torch.float64, device=self.device)
            self.cost = None
        self.tree.load_device(full, [n])
        self.tree.build()
        order = torch.empty(n, dtype=torch.int32, device=self.device)
        self.tree.order_device(order)
        cuts = self.cuts(order, n)
        a, b = cuts[self.rank], cuts[self.rank + 1]
        m = b - a
        active = order[a:b].contiguous()
        acc_m = torch.empty((max(m, 1), 3), dtype=torch.float64, device=self.device)
        pot_m = torch.empty(max(m, 1), dtype=torch.float64, device=self.device)
        nint_m = torch.zeros(max(m, 1), dtype=torch.int32, device=self.device)
        if m:
            self.tree.evaluate_device(acc_m, pot_m, d_active=active, n_active=m,
                                      d_old_acc=self.oldacc if have_old else None,
                                      err_tol_force_acc=err_tol_force_acc, err_tol_theta=err_tol_theta,
                                      d_ninter=nint_m)
        rows = torch.cat([acc_m[:m], pot_m[:m, None], nint_m[:m, None].double()], dim=1)
        sizes = [cuts[r + 1] - cuts[r] for r in range(self.world)]
        res_sorted = self._all_gather_rows(rows, sizes)           # sorted positions 0..n-1
        res = torch.empty_like(res_sorted)
        res[order.long()] = res_sorted                           # back to gathered load order
        d_acc.copy_(res[off:off + n_local, :3])
        d_pot.copy_(res[off:off + n_local, 3])
        self.oldacc = torch.linalg.norm(res[:, :3], dim=1).contiguous()
        self.cost = res[:, 4].contiguous()
        self.kept_counts = list(counts)
        self.last_cuts = cuts
        return off, n_local
