"""The multi-rank host path, world size 2, gloo on CPU."""
import os
import socket

import numpy as np
import pytest

import multi


def test_assign_systems_covers_every_system_once_and_balances():
    rng = np.random.default_rng(3)
    counts = np.exp(rng.uniform(np.log(256), np.log(65536), 4096)).astype(np.int64)
    parts = [multi.assign_systems(counts, 4, r) for r in range(4)]
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(4096))
    loads = [counts[p].sum() for p in parts]
    assert max(loads) / min(loads) < 1.01
    assert multi.rank_seed(10, 0) == 10 and multi.rank_seed(10, 1) != multi.rank_seed(10, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, size, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(size), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import ics
    dist = multi.init("gloo", timeout_s=60)
    counts = np.array([5000, 300, 2000, 1200, 900, 4000], dtype=np.int64)
    mine = multi.assign_systems(counts, size, rank)
    # each rank generates and "evaluates" its own systems: here the number of particles it owns
    n_mine = int(sum(ics.plummer(int(counts[s]), seed=multi.rank_seed(100, s))["pos"].shape[0] for s in mine))
    total = multi.sum_over_ranks(dist, n_mine)
    slowest = multi.max_over_ranks(dist, 1.0 + rank)
    dist.barrier()
    q.put((rank, sorted(mine.tolist()), n_mine, total, slowest))
    dist.destroy_process_group()


def test_two_gloo_ranks_partition_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, n0, t0, m0), (r1, s1, n1, t1, m1) = res
    assert sorted(s0 + s1) == list(range(6)) and not set(s0) & set(s1)
    assert t0 == t1 == n0 + n1 == 13400
    assert m0 == m1 == 2.0


class _FakeTree:
    """Stand-in for the library context: records what a rank loads and walks.
    Its "Peano-Hilbert" order is the order of the x coordinate; a walked
    target's result names the particle (x position in acc[:, 0], load index
    as the potential) and its interaction count is a fixed function of the
    load index, so that the second step's work-balanced cut is predictable."""

    def __init__(self):
        self.loaded = None
        self.walked = []
        self.old = []

    def _x(self):
        import torch
        rec = self.loaded[0].view(-1, 32)
        return rec[:, :8].contiguous().view(-1).view(dtype=torch.float64)

    def load_device(self, records, counts):
        self.loaded = (records.clone(), list(counts))

    def build(self):
        pass

    def order_device(self, d_order):
        import torch
        d_order[:] = torch.argsort(self._x(), stable=True).to(torch.int32)

    def evaluate_device(self, d_acc, d_pot, d_active=None, n_active=0, d_old_acc=None, err_tol_force_acc=0.0,
                        err_tol_theta=0.0, d_ninter=None):
        act = d_active.long()
        self.walked.append(act.clone())
        self.old.append(None if d_old_acc is None else d_old_acc.clone())
        d_acc[:n_active, 0] = self._x()[act]
        d_acc[:n_active, 1:] = 0.0
        d_pot[:n_active] = act.double()
        d_ninter[:n_active] = (act % 7 + 1).to(d_ninter.dtype)


def _split_worker(rank, size, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(size), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch
    import ggb200
    dist = multi.init("gloo", timeout_s=60)
    counts = [700, 1300]                                  # uneven shares of one system
    n = sum(counts)
    rng = np.random.default_rng(5)
    pos = rng.normal(size=(n, 3))
    rec = ggb200.make_records(pos, np.full(n, 1e-3), np.full(n, 0.01))
    off = sum(counts[:rank])
    mine = torch.from_numpy(rec[off:off + counts[rank]].view(np.uint8).copy())
    tree = _FakeTree()
    split = multi.SplitSystem(dist, tree, torch, "cpu")
    acc = torch.zeros((counts[rank], 3), dtype=torch.float64)
    pot = torch.zeros(counts[rank], dtype=torch.float64)
    out = {}
    o, m = split.step(mine, acc, pot)
    out["first"] = (o, m, split.tree.loaded[1], split.last_cuts)
    out["full"] = bool(np.array_equal(tree.loaded[0].numpy(), rec.view(np.uint8).reshape(-1)))
    order = np.argsort(pos[:, 0], kind="stable")
    cuts = split.last_cuts
    out["walked_range"] = bool(np.array_equal(tree.walked[0].numpy(), order[cuts[rank]:cuts[rank + 1]]))
    out["own"] = bool(np.array_equal(acc[:, 0].numpy(), pos[off:off + counts[rank], 0]) and
                      np.array_equal(pot.numpy(), np.arange(off, off + counts[rank])))
    out["no_old_first"] = tree.old[0] is None
    # second step: OldAcc of every particle (|a| of the first step) and a cut
    # that splits the cumulative cost (interactions + 1) along the order in two
    split.step(mine, acc, pot)
    cost = (np.arange(n) % 7 + 1 + 1).astype(np.float64)[order]
    cum = np.cumsum(cost)
    expect = [0, int(np.searchsorted(cum, cum[-1] / 2)), n]
    out["balanced_cut"] = (split.last_cuts, expect)
    out["old_second"] = bool(tree.old[1] is not None and np.allclose(tree.old[1].numpy(), np.abs(pos[:, 0])))
    out["own2"] = bool(np.array_equal(acc[:, 0].numpy(), pos[off:off + counts[rank], 0]))
    # shares of other sizes: the kept OldAcc would name other particles, so it is dropped
    sizes = [900, 1100]
    off2 = sum(sizes[:rank])
    mine2 = torch.from_numpy(rec[off2:off2 + sizes[rank]].view(np.uint8).copy())
    acc2 = torch.zeros((sizes[rank], 3), dtype=torch.float64)
    pot2 = torch.zeros(sizes[rank], dtype=torch.float64)
    split.step(mine2, acc2, pot2)
    out["old_dropped"] = tree.old[2] is None and split.last_cuts == [0, n // 2, n]
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def test_split_system_walks_peano_hilbert_ranges_balanced_by_cost():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    o0, n0, c0, cuts0 = res[0]["first"]
    o1, n1, c1, cuts1 = res[1]["first"]
    assert (o0, n0, o1, n1) == (0, 700, 700, 1300) and c0 == c1 == [2000]
    assert cuts0 == cuts1 == [0, 1000, 2000]              # equal ranges before any cost is known
    for r in (0, 1):
        d = res[r]
        assert d["full"] and d["walked_range"] and d["own"] and d["no_old_first"], (r, d)
        got, expect = d["balanced_cut"]
        assert got == expect, (r, got, expect)
        assert d["old_second"] and d["own2"] and d["old_dropped"], (r, d)
