"""CPU checks of the oracle (FP64 restatement of GIZMO's tree gravity)."""
import numpy as np
import pytest

import ics
import oracle


def test_kernel_known_answers():
    # KERNEL_FAC_FROM_FORCESOFT_TO_PLUMMER = -1/kernel_gravity(0,1,1,-1) = 1/2.8 (kernel.h:709)
    assert oracle.spline_gravity(0.0, 1.0, 1.0, -1) == pytest.approx(-2.8, abs=1e-12)
    # continuity of force and potential factors at u = 0.5 and u = 1 (kernel.h:452-470)
    for mode in (1, -1):
        for u in (0.5, 1.0):
            lo = oracle.spline_gravity(u - 1e-9, 1.0, 1.0, mode)
            hi = oracle.spline_gravity(u + 1e-9, 1.0, 1.0, mode)
            assert lo == pytest.approx(hi, rel=1e-6, abs=1e-6)
    # Newtonian outside the kernel
    assert oracle.spline_gravity(2.0, 1.0, 1.0, 1) == pytest.approx(1 / 8.0)
    assert oracle.spline_gravity(2.0, 1.0, 1.0, -1) == pytest.approx(-0.5)


def test_extent_matches_definition():
    rng = np.random.default_rng(1)
    pos = rng.normal(size=(1000, 3)) * [1, 2, 3]
    d = oracle.find_extent(pos)
    ext = pos.max(0) - pos.min(0)
    assert d["len"] == pytest.approx(1.001 * ext.max(), rel=1e-15)
    assert np.allclose(d["center"], 0.5 * (pos.max(0) + pos.min(0)), rtol=0, atol=1e-15)
    assert np.allclose(np.array(d["corner"]), np.array(d["center"]) - 0.5 * d["len"], atol=1e-15)


def test_key_depth_identity():
    """The 21-bit key is the 42-bit key shifted right by 63 (MSB-first key, peano.c:309-316)."""
    rng = np.random.default_rng(2)
    pos = rng.uniform(-1, 1, size=(5000, 3))
    d = oracle.find_extent(pos)
    hi42, lo42 = oracle.ph_keys(pos, d, bits=42)
    hi21, lo21 = oracle.ph_keys(pos, d, bits=21)
    k42 = [(int(h) << 64) | int(l) for h, l in zip(hi42, lo42)]
    k21 = [(int(h) << 64) | int(l) for h, l in zip(hi21, lo21)]
    assert all(a >> 63 == b for a, b in zip(k42, k21))


def test_key_generator_table_matches_oracle():
    """The packed state table used by the CUDA key kernel gives the oracle's keys."""
    import gen_ph_tables as g
    table = g.build_table()
    table2 = g.build_table2(table)   # two levels per step, as the kernel walks it
    rng = np.random.default_rng(3)
    pos = rng.uniform(-5, 5, size=(3000, 3))
    d = oracle.find_extent(pos)
    hi, lo = oracle.ph_keys(pos, d, bits=21)
    L = oracle.lib()
    for i in range(pos.shape[0]):
        q = [int(L.oracle_double_to_int(((pos[i, j] - d["corner"][j]) / d["len"]) + 1.0, 21)) for j in range(3)]
        assert g.key_python(q[0], q[1], q[2], 21, table) == (int(hi[i]) << 64 | int(lo[i]))
        assert g.key_python2(q[0], q[1], q[2], 21, table, table2) == (int(hi[i]) << 64 | int(lo[i]))


def test_direct_sum_conserves_momentum():
    ic = ics.plummer(2000, seed=7)
    acc, pot = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"])
    p = (ic["mass"][:, None] * acc).sum(0)
    assert np.abs(p).max() < 1e-12 * np.abs(ic["mass"][:, None] * acc).sum()


def test_tree_with_zero_tolerance_is_direct_sum():
    """Relative criterion with OldAcc = 0 opens every node: the walk sums every particle."""
    ic = ics.plummer(1500, seed=8)
    acc_t, pot_t, nint, total = oracle.tree_gravity(ic["pos"], ic["mass"], ic["h"], np.zeros(1500), 0.0025, 0.0)
    acc_d, pot_d = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"])
    assert np.all(nint == 1499)
    assert np.allclose(acc_t, acc_d, rtol=1e-12, atol=1e-12 * np.abs(acc_d).max())
    assert np.allclose(pot_t, pot_d, rtol=1e-12)


def test_tree_error_is_small_and_shrinks_with_tolerance():
    ic = ics.plummer(4096, seed=9)
    acc_d, _ = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"])
    acc1, _, _, tot1, _ = oracle.tree_gravity_two_pass(ic["pos"], ic["mass"], ic["h"], 0.005)
    acc2, _, _, tot2, _ = oracle.tree_gravity_two_pass(ic["pos"], ic["mass"], ic["h"], 0.0005)
    e1 = ics.error_stats(acc1, acc_d)
    e2 = ics.error_stats(acc2, acc_d)
    assert e1[1] < 0.02 and e2[1] < e1[1] and tot2 > tot1


def test_plummer_generator_shape():
    ic = ics.plummer(10000, seed=11)
    r = np.linalg.norm(ic["pos"], axis=1)
    assert r.max() <= 20.0
    # half-mass radius of a Plummer sphere (truncation at 20a shifts it by < 1%)
    assert np.median(r) == pytest.approx(1.0 / np.sqrt(2 ** (2 / 3) - 1), rel=0.05)
    assert ic["h"][0] == pytest.approx(0.028)
