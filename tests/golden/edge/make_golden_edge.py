#!/usr/bin/env python3
"""Golden vectors for degenerate inputs, produced by the reference code itself.

Runs oracle/_ref/gizmo_ref (GIZMO's own sources, one OpenMP thread so that its
interaction counter is exact) on two seeded 600-particle Plummer spheres:

  duplicates_630: 30 particles repeated at exactly the same position (and
      mass and softening).  Coincident pairs have r = 0: they exert no force
      on each other and are not counted (forcetree.c:2258).
  massless_600: 20 particles with zero mass.  GIZMO removes zero-mass
      particles in rearrange_particle_sequence (merge_split.c:1180-1188),
      called before every tree build (domain.c:118), so the reference walks
      and reports only the 580 massive ones; the file keeps which.
  sheet_600: every particle at z = 0 (a flat root cube content).
  two_2: two particles.
  lattice_512: an 8x8x8 lattice, so keys tie at every level down to the
      lattice spacing.
(A one-particle system stops the reference itself: MPI_Abort(11).)
  active_10pct_2000: a clustered system of 2,000 particles in which a
      seeded 10% are active: both start-up passes walk only those (the
      harness's sample-only mode sets GIZMO's active list), with the tree
      built from all particles.
  active_drift_2000: the same system, all particles active at start-up,
      then a drift of DRIFT_DT without a rebuild after which only a seeded
      10% are active (force_drift_node inside the reference's walk).

Stores the inputs, the reference's Barnes-Hut and relative passes (GravAccel,
Potential with G = 1, interaction counts), the potential-only walk
(compute_potential, from the build variant without EVALPOTENTIAL) with the
OldAcc it used, and the mask of the particles the reference kept.  Requires the reference source
tree, so it runs only where that tree exists; the .npz files it writes are
committed.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "gizmo-public_b200")]

import ics  # noqa: E402
import ref_runner  # noqa: E402

TOL = 0.0025
DRIFT_DT = 0.005


def cases():
    ic = ics.plummer(600, seed=211)
    rng = np.random.default_rng(212)
    dup = rng.choice(600, 30, replace=False)
    yield "duplicates_630", {k: np.concatenate([ic[k], ic[k][dup]]) for k in ("pos", "vel", "mass", "h")}
    zero = rng.choice(600, 20, replace=False)
    m = ic["mass"].copy()
    m[zero] = 0.0
    yield "massless_600", dict(pos=ic["pos"], vel=ic["vel"], mass=m, h=ic["h"])
    ic2 = ics.plummer(600, seed=221)
    flat = ic2["pos"].copy()
    flat[:, 2] = 0.0
    yield "sheet_600", dict(pos=flat, vel=np.zeros_like(flat), mass=ic2["mass"], h=ic2["h"])
    yield "two_2", dict(pos=ic2["pos"][:2].copy(), vel=np.zeros((2, 3)), mass=ic2["mass"][:2] * 300,
                        h=ic2["h"][:2].copy())
    g = np.arange(8, dtype=float)
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) * 0.25
    n = lat.shape[0]
    yield "lattice_512", dict(pos=lat, vel=np.zeros_like(lat), mass=np.full(n, 1.0 / n), h=np.full(n, 0.028))


def main():
    for name, ic in cases():
        r = ref_runner.run(ic, tol=TOL, threads=1)
        rp = ref_runner.run(ic, tol=TOL, threads=1, binary=ref_runner.BIN_POT)   # compute_potential
        s = r["info"]["startup"]
        kept = ic["mass"] > 0
        assert int(s["n"]) == int(kept.sum())
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), pos=ic["pos"], mass=ic["mass"], h=ic["h"], tol=TOL, kept=kept,
            acc_bh=r["acc_bh"][kept], pot_bh=r["pot_bh"][kept], acc=r["acc"][kept], pot=r["pot"][kept],
            cost_bh=s["cost_bh"], cost_rel=s["cost_rel"], pot_only=rp["pot_only"][kept],
            oldacc_pot=rp["oldacc"][kept])
        print(name, "n=%d kept=%d cost_bh=%d cost_rel=%d" % (kept.size, kept.sum(), s["cost_bh"], s["cost_rel"]))


def active_case():
    ic = ics.clustered(2000, seed=231, n_clumps=10)
    act = ics.random_active(2000, 0.1, seed=232)
    r = ref_runner.run(ic, tol=TOL, threads=1, sample=act, sample_only=True)
    s = r["info"]["startup"]
    np.savez_compressed(
        os.path.join(HERE, "active_10pct_2000.npz"), pos=ic["pos"], mass=ic["mass"], h=ic["h"], tol=TOL,
        active=act, acc_bh=r["acc_bh"][act], acc=r["acc"][act], pot=r["pot"][act], cost_bh=s["cost_bh"],
        cost_rel=s["cost_rel"])
    print("active_10pct_2000 active=%d cost_bh=%d cost_rel=%d" % (act.size, s["cost_bh"], s["cost_rel"]))


def active_drift_case():
    ic = ics.clustered(2000, seed=231, n_clumps=10)
    act = ics.random_active(2000, 0.1, seed=233)
    r = ref_runner.run(ic, tol=TOL, threads=1, sample=act, drift_dt=DRIFT_DT)
    dr = r["info"]["drift"]
    np.savez_compressed(
        os.path.join(HERE, "active_drift_2000.npz"), pos=ic["pos"], vel=ic["vel"], mass=ic["mass"], h=ic["h"],
        tol=TOL, active=act, drift_dt=dr["dt"], pos_drift=r["pos_drift"][act], acc_drift=r["acc_drift"][act],
        pot_drift=r["pot_drift"][act], cost_drift=dr["cost"])
    print("active_drift_2000 active=%d cost_drift=%d" % (act.size, dr["cost"]))


if __name__ == "__main__":
    main()
    active_case()
    active_drift_case()
