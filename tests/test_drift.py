"""Re-evaluation of a resident tree after a drift, without a rebuild.

The CUDA drift (gg_load_velocities + gg_drift / gg_drift_systems) against the
oracle's restatement of drift_particle and force_drift_node, which is itself
pinned to the reference's drifted walk by the golden vectors.
"""
import numpy as np
import pytest

import ggb200
import ics
import oracle

pytestmark = pytest.mark.gpu


def _old(ic):
    a, _, _, _, _ = oracle.tree_gravity_two_pass(ic["pos"], ic["mass"], ic["h"], 0.0025)
    return np.linalg.norm(a, axis=1)


@pytest.mark.parametrize("dt", [1e-3, 2e-2])
def test_exact_mode_drift_matches_oracle(dt):
    ic = ics.plummer(4096, seed=301)
    old = _old(ic)
    a_o, p_o, n_o, tot_o, _ = oracle.tree_gravity_drift(ic["pos"], ic["vel"], ic["mass"], ic["h"], dt, old_acc=old)
    with ggb200.GravityTree(leaf_size=1, group_size=1) as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.load_velocities(ic["vel"])
        t.build()
        t.drift(dt)
        a, p, n, st = t.evaluate(old_acc=old, want_ninter=True)
    mism = np.count_nonzero(n != n_o)
    assert mism <= 3, (mism, np.abs(n - n_o).max())
    assert abs(st["interactions"] - tot_o) <= 12
    ok = n == n_o
    rel = np.linalg.norm(a - a_o, axis=1) / np.linalg.norm(a_o, axis=1)
    assert np.percentile(rel[ok], 99) < 2e-5 and rel[ok].max() < 2e-4
    assert np.allclose(p[ok], p_o[ok], rtol=2e-5)


def test_zero_drift_changes_nothing_and_drifts_accumulate():
    ic = ics.plummer(6000, seed=302)
    old = _old(ic)
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.load_velocities(ic["vel"])
        t.build()
        a0, p0, n0, _ = t.evaluate(old_acc=old, want_ninter=True)
        t.drift(0.0)
        a1, p1, n1, _ = t.evaluate(old_acc=old, want_ninter=True)
        t.drift(0.004)
        a2, _, _, _ = t.evaluate(old_acc=old)
    with ggb200.GravityTree() as u:
        u.load(ic["pos"], ic["mass"], ic["h"])
        u.load_velocities(ic["vel"])
        u.build()
        u.drift(0.001)
        u.drift(0.003)
        a3, _, _, _ = u.evaluate(old_acc=old)
    assert np.array_equal(a0, a1) and np.array_equal(p0, p1) and np.array_equal(n0, n1)
    # two drifts adding up to one: the same up to the rounding of the node centres
    rel = np.linalg.norm(a3 - a2, axis=1) / np.linalg.norm(a2, axis=1)
    assert np.percentile(rel, 99) < 1e-5


def test_per_system_drift_equals_each_system_alone():
    a = ics.plummer(3000, seed=303)
    b = ics.plummer(2000, seed=304)
    b["pos"] = b["pos"] * 0.5 + 4.0
    oa, ob = _old(a), _old(b)
    alone = []
    for ic, o, dt in ((a, oa, 0.0), (b, ob, 0.01)):
        with ggb200.GravityTree() as t:
            t.load(ic["pos"], ic["mass"], ic["h"])
            t.load_velocities(ic["vel"])
            t.build()
            if dt:
                t.drift(dt)
            alone.append(t.evaluate(old_acc=o, want_ninter=True))
    with ggb200.GravityTree() as t:
        t.load(np.concatenate([a["pos"], b["pos"]]), np.concatenate([a["mass"], b["mass"]]),
               np.concatenate([a["h"], b["h"]]), counts=[3000, 2000])
        t.load_velocities(np.concatenate([a["vel"], b["vel"]]))
        t.build()
        t.drift([0.0, 0.01])
        acc, pot, nint, _ = t.evaluate(old_acc=np.concatenate([oa, ob]), want_ninter=True)
    assert np.array_equal(acc[:3000], alone[0][0]) and np.array_equal(acc[3000:], alone[1][0])
    assert np.array_equal(pot[3000:], alone[1][1]) and np.array_equal(nint[3000:], alone[1][2])


def test_rebuild_after_drift_equals_build_at_drifted_positions():
    ic = ics.plummer(5000, seed=305)
    dt = 0.01
    moved = ic["pos"] + ic["vel"] * dt   # separate roundings, as the device drift
    old = _old(ic)
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.load_velocities(ic["vel"])
        t.build()
        t.drift(dt)
        t.build()
        a1, p1, n1, _ = t.evaluate(old_acc=old, want_ninter=True)
    with ggb200.GravityTree() as u:
        u.load(moved, ic["mass"], ic["h"])
        u.build()
        a2, p2, n2, _ = u.evaluate(old_acc=old, want_ninter=True)
    assert np.array_equal(a1, a2) and np.array_equal(p1, p2) and np.array_equal(n1, n2)


def test_drift_rejects_missing_state_and_bad_steps():
    ic = ics.plummer(1000, seed=306)
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.load_velocities(ic["vel"])
        with pytest.raises(ggb200.GravityError):
            t.drift(0.01)                 # no tree yet
        t.build()
        with pytest.raises(ggb200.GravityError):
            t.drift(float("nan"))
        t.load(ic["pos"], ic["mass"], ic["h"])   # a new load drops the velocities
        t.build()
        with pytest.raises(ggb200.GravityError):
            t.drift(0.01)


def test_set_positions_with_the_drifted_positions_changes_nothing():
    """gg_set_positions with the positions gg_drift computes (x + v*dt, each
    operation rounded) leaves every result bitwise as it was."""
    ic = ics.plummer(5000, seed=311)
    old = _old(ic)
    dt = 0.003
    res = []
    for reload in (False, True):
        with ggb200.GravityTree() as t:
            t.load(ic["pos"], ic["mass"], ic["h"])
            t.load_velocities(ic["vel"])
            t.build()
            t.drift(dt)
            if reload:
                t.set_positions(ic["pos"] + ic["vel"] * dt)
            res.append(t.evaluate(old_acc=old, want_ninter=True))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    assert np.array_equal(res[0][2], res[1][2])


def test_set_positions_are_the_positions_the_walk_reads():
    """Particles that moved by another rule than Vel*dt (as GIZMO's MFV cells
    do): after gg_drift the caller's positions replace them, for targets and
    sources alike.  With every node opened (relative criterion, OldAcc 0) the
    walk is a direct sum at the caller's positions."""
    ic = ics.plummer(3000, seed=312)
    dt = 0.01
    rng = np.random.default_rng(313)
    moved = ic["pos"] + ic["vel"] * dt
    odd = rng.random(3000) < 0.2
    moved[odd] += rng.normal(scale=0.02, size=(int(odd.sum()), 3))
    acc_d, _ = oracle.direct_sum(moved, ic["mass"], ic["h"])
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.load_velocities(ic["vel"])
        t.build()
        t.drift(dt)
        t.set_positions(moved)
        a, _, _, st = t.evaluate(old_acc=np.zeros(3000), err_tol_theta=0.0)
    assert st["error_word"] == 0
    assert np.allclose(a, acc_d, rtol=1e-4, atol=1e-6 * np.abs(acc_d).max())


def test_set_positions_refuses_non_finite():
    ic = ics.plummer(1000, seed=314)
    bad = ic["pos"].copy()
    bad[7, 2] = np.inf
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.build()
        t.set_positions(bad)
        with pytest.raises(ggb200.GravityError) as ei:
            t.evaluate(err_tol_theta=0.7)
        assert ei.value.status == -7
