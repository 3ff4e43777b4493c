"""One system split over two ranks with real library contexts (multi.SplitSystem).

Two processes (gloo process group, results exchanged through host memory) on
the same GPU, each with its own context; no kernel waits on another process.
Uneven shares of one Plummer sphere: every rank gathers all records, builds
the whole tree and walks one Peano-Hilbert range of targets.  The first
(Barnes-Hut) step cuts the order in equal halves, the second (relative) step
by the first step's costs.  A rank's walk groups are bounded by the tree nodes
holding at most 64 groups of its own targets, so next to a cut they differ
from those of one process walking the whole system.  On both steps the
median and 99th-percentile force errors against the FP64 direct sum stay
within 1.1x those of the plain walk.  On the relative step they also meet the
library's bar against the reference tree (the oracle's restatement of it):
median and 99th percentile within 1.1x, and the potential energy no further
from the direct sum than the reference tree's (or within 1e-5).
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, SHARES = 8192, (3000, 5192)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK="0")
    import torch
    import ggb200
    import ics
    import multi
    dist = multi.init("gloo", timeout_s=120)
    ic = ics.plummer(N, seed=401)
    rec = ggb200.make_records(ic["pos"], ic["mass"], ic["h"])
    off = sum(SHARES[:rank])
    mine = torch.from_numpy(rec[off:off + SHARES[rank]].view(np.uint8).copy()).cuda()
    stream = torch.cuda.Stream()
    out = {}
    with torch.cuda.stream(stream):
        t = ggb200.GravityTree()
        t.set_stream(stream.cuda_stream)
        split = multi.SplitSystem(dist, t, torch, "cuda")
        acc = torch.empty((SHARES[rank], 3), dtype=torch.float64, device="cuda")
        pot = torch.empty(SHARES[rank], dtype=torch.float64, device="cuda")
        split.step(mine, acc, pot, err_tol_theta=0.7)
        torch.cuda.synchronize()
        out["bh"] = (acc.cpu().numpy(), pot.cpu().numpy(), list(split.last_cuts))
        split.step(mine, acc, pot, err_tol_force_acc=0.0025)
        torch.cuda.synchronize()
        out["rel"] = (acc.cpu().numpy(), pot.cpu().numpy(), list(split.last_cuts))
        t.close()
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_on_real_contexts_stay_within_the_plain_walks_error():
    import torch.multiprocessing as mp
    import ggb200
    import ics
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ic = ics.plummer(N, seed=401)
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.build()
        a1, p1, _, _ = t.evaluate(err_tol_theta=0.7)
        a2, p2, _, _ = t.evaluate(old_acc=np.linalg.norm(a1, axis=1), err_tol_force_acc=0.0025)
    acc_d, pot_d = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"])
    m = ic["mass"]
    Wd = 0.5 * np.sum(m * pot_d)

    def within(acc_s, pot_s, acc_p, pot_p, what, energy=False):
        s50, s99, _ = ics.error_stats(acc_s, acc_d)
        q50, q99, _ = ics.error_stats(acc_p, acc_d)
        assert s50 <= 1.1 * q50 and s99 <= 1.1 * q99, (what, s50, s99, q50, q99)
        if energy:
            Ws, Wp = 0.5 * np.sum(m * pot_s), 0.5 * np.sum(m * pot_p)
            assert abs(Ws - Wd) <= max(abs(Wp - Wd), 1e-5 * abs(Wd)), (what, Ws, Wp, Wd)

    assert res[0]["bh"][2] == res[1]["bh"][2] == [0, N // 2, N]
    within(np.concatenate([res[0]["bh"][0], res[1]["bh"][0]]), np.concatenate([res[0]["bh"][1], res[1]["bh"][1]]),
           a1, p1, "Barnes-Hut step vs plain walk")
    cuts = res[0]["rel"][2]
    assert cuts == res[1]["rel"][2] and 0 < cuts[1] < N
    acc_rel = np.concatenate([res[0]["rel"][0], res[1]["rel"][0]])
    pot_rel = np.concatenate([res[0]["rel"][1], res[1]["rel"][1]])
    within(acc_rel, pot_rel, a2, p2, "relative step vs plain walk")
    acc_o, pot_o, _, _, _ = oracle.tree_gravity_two_pass(ic["pos"], ic["mass"], ic["h"], 0.0025)
    within(acc_rel, pot_rel, acc_o, pot_o, "relative step vs reference tree", energy=True)
