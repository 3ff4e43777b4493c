#!/usr/bin/env python3
"""Reference fixtures for the GPU parity tests at the benchmark configurations.

For each configuration below this runs the reference code itself
(oracle/_ref/gizmo_ref: GIZMO's own sources compiled by oracle/build_ref.sh,
OpenMP on every host thread) through its start-up evaluation -- the
Barnes-Hut pass, then the relative pass with ErrTolForceAcc (accel.c:47-50) --
and stores, for a seeded sample of targets (or all of them), the reference
tree's forces and potentials with the FP64 direct sum of the CPU oracle on
the same targets, and the reference tree's median / 99th-percentile relative
force error and sample potential energy against that direct sum.  The initial
conditions are not stored: the tests regenerate them from the seeded
generators in gizmo-public_b200/ics.py and check a few stored positions.

Each target's result in the reference depends only on the tree of all
particles and on its own OldAcc, so one sample serves both the all-active and
the subset walks of the same system.

Requires the reference source tree (to build oracle/_ref), so it runs only
where that tree exists; the .npz files it writes are committed.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "gizmo-public_b200")]

import ics  # noqa: E402
import oracle  # noqa: E402
import ref_runner  # noqa: E402

# the galaxy's halo : disk split (3,000,000 : 1,194,304) at 262,144 particles
GAL_HALO_262K = 187500
GAL_DISK_262K = 262144 - GAL_HALO_262K


def gen(name):
    if name.startswith("plummer_65536"):
        return ics.plummer(65536)
    if name.startswith("galaxy_262144"):
        return ics.galaxy(n_halo=GAL_HALO_262K, n_disk=GAL_DISK_262K)
    if name.startswith("galaxy_4194304"):
        return ics.galaxy()
    if name.startswith("clustered_1048576"):
        return ics.clustered(1048576)
    if name.startswith("clustered_16777216"):
        return ics.clustered()
    raise KeyError(name)


# name -> (ErrTolForceAcc, sample size or None for all, sample seed, active fraction of the subset run)
CASES = {
    "plummer_65536_tol0025": (0.0025, None, 0, 0.0),
    "galaxy_262144_tol0025": (0.0025, 4096, 11, 0.0),
    "galaxy_262144_tol005": (0.005, 4096, 11, 0.0),
    "galaxy_4194304_tol001": (0.001, 4096, 12, 0.0),
    "galaxy_4194304_tol0025": (0.0025, 4096, 12, 0.0),
    "galaxy_4194304_tol005": (0.005, 4096, 12, 0.0),
    "clustered_1048576_tol0025": (0.0025, 4096, 13, 0.1),
    "clustered_1048576_tol0008": (0.0008, 4096, 13, 0.1),
    "clustered_16777216_tol0008": (0.0008, 2048, 14, 0.1),
    "clustered_16777216_tol0025": (0.0025, 2048, 14, 0.1),
}
ACTIVE_SEED = 77


def sample_targets(n, size, seed, frac):
    """Seeded targets; with an active fraction they are drawn from the seeded
    active set (ics.random_active(n, frac, ACTIVE_SEED)), so that the same
    targets belong to both the all-active and the subset walk."""
    if size is None:
        return np.arange(n, dtype=np.int32)
    pool = ics.random_active(n, frac, ACTIVE_SEED) if frac > 0 else np.arange(n, dtype=np.int32)
    pick = np.sort(np.random.default_rng(seed).choice(pool.size, size, replace=False))
    return pool[pick].astype(np.int32)


def make(name):
    tol, size, seed, frac = CASES[name]
    ic = gen(name)
    n = ic["pos"].shape[0]
    tg = sample_targets(n, size, seed, frac)
    t0 = time.time()
    r = ref_runner.run(ic, tol=tol, sample=None if size is None else tg, sample_only=size is not None)
    t1 = time.time()
    acc_ref, pot_ref = r["acc"][tg], r["pot"][tg]
    acc_dir, pot_dir = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"], targets=None if size is None else tg)
    t2 = time.time()
    p50, p99, _ = ics.error_stats(acc_ref, acc_dir)
    m = ic["mass"][tg]
    w_ref, w_dir = 0.5 * np.sum(m * pot_ref), 0.5 * np.sum(m * pot_dir)
    keep = tg if size is not None else tg[:: max(1, n // 4096)]   # forces stored for at most ~4096 targets
    rows = np.searchsorted(tg, keep)
    check = np.linspace(0, n - 1, 16).astype(np.int64)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), n=n, tol=tol, targets=tg if size is not None else np.zeros(0, np.int32),
        all_targets=size is None, active_frac=frac, active_seed=ACTIVE_SEED,
        ref_p50=p50, ref_p99=p99, ref_W=w_ref, direct_W=w_dir,
        kept=keep.astype(np.int32), acc_ref=acc_ref[rows], pot_ref=pot_ref[rows], acc_dir=acc_dir[rows],
        pot_dir=pot_dir[rows], pos_check_idx=check, pos_check=ic["pos"][check],
        ref_cost_rel=r["info"]["startup"]["cost_rel"], ref_threads=r["info"]["startup"]["threads"])
    print("%s n=%d targets=%d ref p50=%.3e p99=%.3e W_ref-W_dir=%.2e (ref %.0fs, direct %.0fs)" % (
        name, n, tg.size, p50, p99, (w_ref - w_dir) / abs(w_dir), t1 - t0, t2 - t1), flush=True)


def main():
    names = sys.argv[1:] or list(CASES)
    for name in names:
        make(name)


if __name__ == "__main__":
    main()
