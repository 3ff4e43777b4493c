"""Degenerate inputs pinned to the reference code itself
(tests/golden/edge/make_golden_edge.py).

Exact duplicates, a flat sheet, two particles and a lattice whose keys tie
down to its spacing: the oracle reproduces the reference's interaction counts
exactly and its forces and potentials to FP64 rounding (coincident particles
exert no force on each other and are not counted).  Massless particles: GIZMO removes
them before every tree build (merge_split.c:1180-1188), so its outputs cover
the massive particles only; the oracle reproduces them on that subset, and,
with the massless particles left in, ignores them as sources (the massive
particles' forces do not change) while still giving them a finite force.
"""
import glob
import os

import numpy as np
import pytest

import oracle

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "edge")


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    return {k: z[k] for k in z.files}


def two_pass(pos, mass, h, tol):
    a1, p1, _, c1 = oracle.tree_gravity(pos, mass, h, None, tol, 0.7)
    a2, p2, _, c2 = oracle.tree_gravity(pos, mass, h, np.linalg.norm(a1, axis=1), tol, 0.0)
    return a1, p1, c1, a2, p2, c2


def close(a, b):
    return np.allclose(a, b, rtol=1e-12, atol=1e-14 * np.abs(b).max())


def test_fixtures_present():
    assert sorted(os.path.basename(p) for p in glob.glob(os.path.join(HERE, "*.npz"))) == [
        "active_10pct_2000.npz", "active_drift_2000.npz", "duplicates_630.npz", "lattice_512.npz", "massless_600.npz", "sheet_600.npz",
        "two_2.npz"]


@pytest.mark.parametrize("name", ["sheet_600", "two_2", "lattice_512"])
def test_degenerate_shapes_match_reference(name):
    g = load(name)
    assert g["kept"].all()
    a1, p1, c1, a2, p2, c2 = two_pass(g["pos"], g["mass"], g["h"], float(g["tol"]))
    assert c1 == int(g["cost_bh"]) and c2 == int(g["cost_rel"])
    assert close(a1, g["acc_bh"]) and close(a2, g["acc"]) and close(p2, g["pot"])


def test_exact_duplicates_match_reference():
    g = load("duplicates_630")
    assert g["kept"].all()
    a1, p1, c1, a2, p2, c2 = two_pass(g["pos"], g["mass"], g["h"], float(g["tol"]))
    assert c1 == int(g["cost_bh"]) and c2 == int(g["cost_rel"])
    assert close(a1, g["acc_bh"]) and close(a2, g["acc"]) and close(p2, g["pot"])
    # the duplicated particles feel the same force as their originals
    n0 = g["pos"].shape[0] - 30
    orig = [int(np.flatnonzero((g["pos"][:n0] == g["pos"][i]).all(axis=1))[0]) for i in range(n0, n0 + 30)]
    assert np.array_equal(a2[n0:], a2[orig])


def test_massless_particles_reference_keeps_only_massive():
    g = load("massless_600")
    k = g["kept"]
    assert k.sum() == 580 and np.all(g["mass"][k] > 0) and np.all(g["mass"][~k] == 0)
    a1, p1, c1, a2, p2, c2 = two_pass(g["pos"][k], g["mass"][k], g["h"][k], float(g["tol"]))
    assert c1 == int(g["cost_bh"]) and c2 == int(g["cost_rel"])
    assert close(a1, g["acc_bh"]) and close(a2, g["acc"]) and close(p2, g["pot"])


@pytest.mark.parametrize("tol", [0.0025])
def test_massless_particles_are_ignored_as_sources(tol):
    g = load("massless_600")
    k = g["kept"]
    a1, p1, c1, a2, p2, c2 = two_pass(g["pos"], g["mass"], g["h"], tol)
    assert close(a2[k], g["acc"]) and close(p2[k], g["pot"])
    assert np.isfinite(a2[~k]).all() and (np.linalg.norm(a2[~k], axis=1) > 0).all()
    # only the massless targets' own walks add to the count
    assert c2 > int(g["cost_rel"])


@pytest.mark.parametrize("name", ["duplicates_630", "sheet_600", "two_2", "lattice_512", "massless_600"])
def test_potential_walk_matches_reference(name):
    g = load(name)
    k = g["kept"]
    p = oracle.potential(g["pos"][k], g["mass"][k], g["h"][k], old_acc=g["oldacc_pot"],
                         err_tol_force_acc=float(g["tol"]))
    assert np.allclose(p, g["pot_only"], rtol=1e-12, atol=1e-14 * np.abs(g["pot_only"]).max())


def test_active_subset_matches_reference():
    """GIZMO walks only the active particles on a tree of all of them; the
    Barnes-Hut pass gives the active ones their OldAcc for the relative pass."""
    g = load("active_10pct_2000")
    act, tol = g["active"], float(g["tol"])
    a1, p1, _, c1 = oracle.tree_gravity(g["pos"], g["mass"], g["h"], None, tol, 0.7, targets=act)
    old = np.zeros(g["pos"].shape[0])
    old[act] = np.linalg.norm(a1, axis=1)
    a2, p2, _, c2 = oracle.tree_gravity(g["pos"], g["mass"], g["h"], old, tol, 0.0, targets=act)
    assert c1 == int(g["cost_bh"]) and c2 == int(g["cost_rel"])
    assert close(a1, g["acc_bh"]) and close(a2, g["acc"]) and close(p2, g["pot"])


def test_active_subset_after_drift_matches_reference():
    """Start-up passes over all particles, then a drift without a rebuild and
    a walk of the active 10% only: nodes drifted inside the walk
    (force_drift_node) and the relative criterion on the start-up OldAcc."""
    g = load("active_drift_2000")
    act, tol = g["active"], float(g["tol"])
    a1, _, _, _ = oracle.tree_gravity(g["pos"], g["mass"], g["h"], None, tol, 0.7)
    a2, _, _, _ = oracle.tree_gravity(g["pos"], g["mass"], g["h"], np.linalg.norm(a1, axis=1), tol, 0.0)
    a3, p3, _, c3, moved = oracle.tree_gravity_drift(g["pos"], g["vel"], g["mass"], g["h"], float(g["drift_dt"]),
                                                     np.linalg.norm(a2, axis=1), tol, 0.0, targets=act)
    assert c3 == int(g["cost_drift"])
    assert np.allclose(moved[act], g["pos_drift"], rtol=0, atol=4 * np.spacing(np.abs(g["pos_drift"]).max()))
    assert close(a3, g["acc_drift"]) and close(p3, g["pot_drift"])
