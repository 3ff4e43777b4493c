"""Parity at the benchmark configurations, against the reference's own tree.

Fixtures (tests/golden/config/, made by make_config_golden.py from the
reference code itself) hold, per configuration, the reference tree's forces
and potentials on seeded targets after its start-up evaluation (Barnes-Hut
pass, then the relative pass, accel.c:47-50), the CPU oracle's FP64 direct
sum on the same targets, and the reference tree's median / 99th-percentile
relative error and sample potential energy against it.  The systems are
regenerated from their seeds.

GPU: the default configuration (leaf buckets of 8, groups of 32 targets) runs
the same two passes; its errors against the FP64 direct sum (this library's
k_direct, checked against the oracle's direct sum here too) must be no worse
than 1.1x the reference tree's, median and 99th percentile, and its sample
potential energy no further from the direct sum than the reference's (or
within 1e-5).  Systems with an active fraction are also walked with only that
seeded random subset active (individual timesteps), on the same tree.
CPU: the fixtures are consistent with the oracle and the generators.
"""
import os
import sys

import numpy as np
import pytest

import ggb200
import ics
import oracle

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config")
sys.path.insert(0, HERE)
import make_config_golden as mk  # noqa: E402

SMALL = ["plummer_65536_tol0025", "galaxy_262144_tol0025", "galaxy_262144_tol005", "clustered_1048576_tol0025",
         "clustered_1048576_tol0008"]
# at the benchmark's tolerances: also the metric's bound p99 < 2e-3
FULL = ["galaxy_4194304_tol001", "clustered_16777216_tol0008"]
# at the configurations' own tolerances (the galaxy's 0.0025 and 0.005, the
# clustered system's 0.0025): the reference tree's bound only
FULL_CONFIG = ["galaxy_4194304_tol0025", "galaxy_4194304_tol005", "clustered_16777216_tol0025"]


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    return {k: z[k] for k in z.files}


def targets_of(g):
    return np.arange(int(g["n"]), dtype=np.int32) if bool(g["all_targets"]) else g["targets"].astype(np.int32)


def system(name, g):
    ic = mk.gen(name)
    # the generators are seeded; transcendental functions may differ by a unit
    # in the last place between hosts, far below anything the errors resolve
    assert ic["pos"].shape[0] == int(g["n"])
    assert np.allclose(ic["pos"][g["pos_check_idx"]], g["pos_check"], rtol=1e-12, atol=1e-15)
    return ic


# ---------------------------------------------------------------- CPU
@pytest.mark.parametrize("name", SMALL)
def test_fixture_consistent_with_oracle(name):
    g = load(name)
    ic = system(name, g)
    tg = targets_of(g)
    kept = g["kept"]
    assert np.all(np.isin(kept, tg))
    # the stored direct sum is the oracle's, on a few of the kept targets
    few = kept[:: max(1, kept.size // 8)][:8]
    rows = np.searchsorted(kept, few)
    a, p = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"], targets=few)
    assert np.allclose(a, g["acc_dir"][rows], rtol=1e-12, atol=0) and np.allclose(p, g["pot_dir"][rows], rtol=1e-12)
    if not bool(g["all_targets"]):
        # the stored statistics are those of the stored forces
        r50, r99, _ = ics.error_stats(g["acc_ref"], g["acc_dir"])
        assert r50 == pytest.approx(float(g["ref_p50"]), rel=1e-12)
        assert r99 == pytest.approx(float(g["ref_p99"]), rel=1e-12)
    if float(g["active_frac"]) > 0:
        act = ics.random_active(int(g["n"]), float(g["active_frac"]), int(g["active_seed"]))
        assert np.all(np.isin(tg, act))


# ---------------------------------------------------------------- GPU
def gpu_direct(ic, tg):
    import torch
    n = ic["pos"].shape[0]
    dp, dm, dh = (torch.from_numpy(np.ascontiguousarray(ic[k])).cuda() for k in ("pos", "mass", "h"))
    da = torch.empty((tg.size, 3), dtype=torch.float64, device="cuda")
    dpo = torch.empty(tg.size, dtype=torch.float64, device="cuda")
    ggb200.direct_sum_fp64(dp, dm, dh, n, torch.from_numpy(tg).cuda(), tg.size, da, dpo)
    torch.cuda.synchronize()
    return da.cpu().numpy(), dpo.cpu().numpy()


def check_against_reference(g, ic, tg, acc, pot, acc_dir, pot_dir, what):
    p50, p99, _ = ics.error_stats(acc, acc_dir)
    r50, r99 = float(g["ref_p50"]), float(g["ref_p99"])
    assert p50 <= 1.1 * r50 and p99 <= 1.1 * r99, (what, p50, p99, r50, r99)
    m = ic["mass"][tg]
    W, Wd = 0.5 * np.sum(m * pot), 0.5 * np.sum(m * pot_dir)
    Wr = float(g["ref_W"])
    assert abs(Wd - float(g["direct_W"])) <= 1e-10 * abs(Wd)
    assert abs(W - Wd) <= max(abs(Wr - Wd), 1e-5 * abs(Wd)), (what, W, Wd, Wr)
    return p50, p99


def run_config(name):
    g = load(name)
    ic = system(name, g)
    n, tol = int(g["n"]), float(g["tol"])
    tg = targets_of(g)
    acc_dir, pot_dir = gpu_direct(ic, tg)
    rows = np.searchsorted(tg, g["kept"])
    assert np.allclose(acc_dir[rows], g["acc_dir"], rtol=1e-10, atol=1e-12 * np.abs(g["acc_dir"]).max())
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.build()
        a1, _, _, _ = t.evaluate(err_tol_theta=0.7)
        old = np.linalg.norm(a1, axis=1)
        acc, pot, _, st = t.evaluate(old_acc=old, err_tol_force_acc=tol)
        assert st["error_word"] == 0
        p50, p99 = check_against_reference(g, ic, tg, acc[tg], pot[tg], acc_dir, pot_dir, "all active")
        out = {"p50": p50, "p99": p99}
        if float(g["active_frac"]) > 0:
            act = ics.random_active(n, float(g["active_frac"]), int(g["active_seed"]))
            acc_s, pot_s, _, st = t.evaluate(active=act, old_acc=old, err_tol_force_acc=tol)
            assert st["error_word"] == 0 and st["n_targets"] == act.size
            r = np.searchsorted(act, tg)
            s50, s99 = check_against_reference(g, ic, tg, acc_s[r], pot_s[r], acc_dir, pot_dir, "subset")
            out.update(subset_p50=s50, subset_p99=s99)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", SMALL)
def test_default_walk_within_reference_bound(name):
    run_config(name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", FULL)
def test_full_size_within_reference_bound_and_metric(name):
    """The galaxy (4,194,304) and the clustered system (16,777,216, all active
    and 10% active) at the benchmark's tolerance: no worse than 1.1x the
    reference tree, and p99 below the metric's 2e-3."""
    out = run_config(name)
    assert out["p99"] < 2e-3, out
    if "subset_p99" in out:
        assert out["subset_p99"] < 2e-3, out


@pytest.mark.gpu
@pytest.mark.parametrize("name", FULL_CONFIG)
def test_full_size_within_reference_bound_at_config_tolerance(name):
    run_config(name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["clustered_1048576_tol0008", "clustered_16777216_tol0008", "galaxy_4194304_tol001"])
def test_autotuned_configuration_within_reference_bound(name):
    """The configuration the benchmark times is the gated autotuner's choice
    for the system; it too stays within 1.1x the reference tree."""
    g = load(name)
    ic = system(name, g)
    tol = float(g["tol"])
    tg = targets_of(g)
    acc_dir, pot_dir = gpu_direct(ic, tg)
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.build()
        a1, _, _, _ = t.evaluate(err_tol_theta=0.7)
        old = np.linalg.norm(a1, axis=1)
        t.evaluate(old_acc=old, err_tol_force_acc=tol)
        cfg, _ = t.autotune(err_tol_force_acc=tol)
        t.build()
        acc, pot, _, st = t.evaluate(old_acc=old, err_tol_force_acc=tol)
    assert st["error_word"] == 0
    check_against_reference(g, ic, tg, acc[tg], pot[tg], acc_dir, pot_dir, "tuned %s" % cfg)
