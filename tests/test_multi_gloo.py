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
    """Stand-in for the library context: records what a rank loads and walks."""

    def __init__(self):
        self.loaded = None

    def load_device(self, records, counts):
        self.loaded = (records.clone(), list(counts))

    def build(self):
        pass

    def evaluate_device(self, d_acc, d_pot, d_active=None, n_active=0, d_old_acc=None, err_tol_force_acc=0.0,
                        err_tol_theta=0.0):
        rec = self.loaded[0].view(-1, 32)
        act = d_active.long()
        # a result that names the particle: its first position word
        d_acc[:, 0] = rec[act, :8].contiguous().view(-1).view(dtype=__import__("torch").float64)
        d_pot[:] = act.double()


def _split_worker(rank, size, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(size), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch
    import ggb200
    dist = multi.init("gloo", timeout_s=60)
    counts = [700, 1300]                                  # uneven shares of one system
    rng = np.random.default_rng(5)
    pos = rng.normal(size=(sum(counts), 3))
    rec = ggb200.make_records(pos, np.full(sum(counts), 1e-3), np.full(sum(counts), 0.01))
    off = sum(counts[:rank])
    mine = torch.from_numpy(rec[off:off + counts[rank]].view(np.uint8).copy())
    split = multi.SplitSystem(dist, _FakeTree(), torch, "cpu")
    acc = torch.zeros((counts[rank], 3), dtype=torch.float64)
    pot = torch.zeros(counts[rank], dtype=torch.float64)
    o, n = split.step(mine, acc, pot)
    full = split.tree.loaded[0].numpy()
    ok_full = bool(np.array_equal(full, rec.view(np.uint8).reshape(-1)))
    ok_own = bool(np.array_equal(acc[:, 0].numpy(), pos[off:off + counts[rank], 0]))
    ok_idx = bool(np.array_equal(pot.numpy(), np.arange(off, off + counts[rank])))
    q.put((rank, o, n, split.tree.loaded[1], ok_full, ok_own, ok_idx))
    dist.barrier()
    dist.destroy_process_group()


def test_split_system_gathers_everything_and_walks_only_its_own_particles():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, o0, n0, c0, f0, w0, i0), (r1, o1, n1, c1, f1, w1, i1) = res
    assert (o0, n0, o1, n1) == (0, 700, 700, 1300) and c0 == c1 == [2000]
    assert f0 and f1 and w0 and w1 and i0 and i1
