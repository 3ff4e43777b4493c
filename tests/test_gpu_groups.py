"""Walk groups bounded by tree nodes.

A group never spans two group nodes, the shallowest tree nodes that hold at
most 64 groups' worth of the walk's targets; within a group node the targets
are cut into runs of the group size.  The expected group count is rebuilt here
from the oracle's Peano-Hilbert keys (bitwise those of the library): a tree
node's particles are those of the key-prefix cell at its level, so the group
node of a target is the shallowest prefix cell holding at most 64 x group size
of the walk's targets.  The systems have one kernel radius (targets in key
order) and no two particles in one full-depth cell.

CPU: the restatement on hand-made keys.  GPU: the library's group count for
all targets and for a seeded 10% subset, two group sizes.
"""
import numpy as np
import pytest

import ggb200
import ics
import oracle

LEVELS = 21


def expected_groups(sorted_keys, is_target, gs):
    """Groups of a walk over the targets among the sorted keys (one system)."""
    cap = 64 * gs
    n = sorted_keys.size
    tcum = np.concatenate([[0], np.cumsum(is_target.astype(np.int64))])
    gnode = np.full(n, -1, np.int64)
    for lev in range(LEVELS + 1):
        pre = sorted_keys >> np.uint64(3 * (LEVELS - lev))
        starts = np.flatnonzero(np.r_[True, pre[1:] != pre[:-1]])
        ends = np.r_[starts[1:], n]
        counts = tcum[ends] - tcum[starts]
        run = np.repeat(np.arange(starts.size), ends - starts)
        take = (counts[run] <= cap) & (gnode < 0)
        gnode[take] = (lev << 40) + run[take]
        if (gnode >= 0).all():
            break
    tg = gnode[is_target]
    if tg.size == 0:
        return 0
    seg = np.flatnonzero(np.r_[True, tg[1:] != tg[:-1]])
    seglen = np.diff(np.r_[seg, tg.size])
    return int(np.sum((seglen + gs - 1) // gs))


def test_restatement_on_hand_made_keys():
    # 3 x 64 keys in one level-1 octant, 200 in another: with groups of 1
    # (cap 64) the first octant's 192 split into its three level-2 cells
    k = np.concatenate([np.full(64, 0), np.full(64, 1), np.full(64, 2), np.full(200, 7 << 3)]).astype(np.uint64)
    k = (k << np.uint64(3 * (LEVELS - 2))) + np.arange(k.size, dtype=np.uint64)   # distinct, sorted
    assert np.all(np.diff(k.astype(np.int64)) > 0)
    allt = np.ones(k.size, bool)
    # gs = 1: cap 64 -> cells of 64 (3 groups... of size 1 each: 192 groups) + the 200 split deeper
    assert expected_groups(k, allt, 1) == k.size
    # gs = 4: cap 256 -> the first octant (192) and the second (200) are group nodes: 48 + 50 groups
    assert expected_groups(k, allt, 4) == 48 + 50
    # gs = 64: cap 4096 -> the root: ceil(392 / 64) groups
    assert expected_groups(k, allt, 64) == 7
    # targets only in the second octant: one group node, ceil(200 / 64)
    assert expected_groups(k, np.r_[np.zeros(192, bool), np.ones(200, bool)], 64) == 4


@pytest.mark.gpu
@pytest.mark.parametrize("gs", [32, 64])
def test_group_count_matches_restatement(gs):
    n = 300000
    ic = ics.clustered(n, seed=71, n_clumps=60)
    dom = oracle.find_extent(ic["pos"])
    hi, lo = oracle.ph_keys(ic["pos"], dom)
    assert not hi.any()
    order = np.argsort(lo, kind="stable")
    keys = lo[order]
    # no full-depth cell holds two particles (the library would split it into chunks)
    assert np.all(np.diff(keys.astype(np.int64)) > 0)
    act = ics.random_active(n, 0.1, seed=72)
    is_act = np.zeros(n, bool)
    is_act[act] = True
    with ggb200.GravityTree(group_size=gs) as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.build()
        t.evaluate(err_tol_theta=0.7)
        full = t.last_stats()["n_groups"]
        t.evaluate(active=act, err_tol_theta=0.7)
        sub = t.last_stats()["n_groups"]
    assert full == expected_groups(keys, np.ones(n, bool), gs)
    assert sub == expected_groups(keys, is_act[order], gs)
    assert full > n // gs   # some group nodes end in partial groups
