#!/usr/bin/env python3
"""Generate golden vectors from the reference code itself.

Runs oracle/_ref/gizmo_ref (GIZMO's own sources compiled by oracle/build_ref.sh,
single OpenMP thread so that its interaction counter Costtotal is exact) on
small seeded systems and stores, per case, the inputs and the reference's
outputs: root cube, 42-bit Peano-Hilbert keys (peano_hilbert_key), the
Barnes-Hut pass and the relative pass (GravAccel, Potential; G = 1) and the
interaction counts of both passes; then a re-evaluation after a drift of
DRIFT_DT without a rebuild (drifted positions, forces, potentials and count),
in which GIZMO's walk moves the tree nodes itself (force_drift_node); and
the potential-only walk (compute_potential) of the build variant without
EVALPOTENTIAL, run on the same tree after the start-up passes.  Requires the reference source tree, so it
runs only where that tree exists; the .npz files it writes are committed.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "gizmo-public_b200")]

import ics  # noqa: E402
import ref_runner  # noqa: E402

DRIFT_DT = 0.005

CASES = {
    "plummer_1024": (lambda: ics.plummer(1024, seed=101), 0.0025),
    "galaxy_1500": (lambda: ics.galaxy(n_halo=1070, n_disk=430, seed=102), 0.0025),
    "galaxy_1500_tol005": (lambda: ics.galaxy(n_halo=1070, n_disk=430, seed=102), 0.005),
    "clustered_1500": (lambda: ics.clustered(1500, seed=103, n_clumps=8), 0.0025),
}


def main():
    for name, (gen, tol) in CASES.items():
        ic = gen()
        r = ref_runner.run(ic, tol=tol, threads=1, drift_dt=DRIFT_DT)
        rp = ref_runner.run(ic, tol=tol, threads=1, binary=ref_runner.BIN_POT)
        s = r["info"]["startup"]
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), pos=ic["pos"], mass=ic["mass"], h=ic["h"], tol=tol,
            corner=np.array(r["info"]["domain"]["corner"]), len=r["info"]["domain"]["len"],
            key_hi=r["key_hi"], key_lo=r["key_lo"], acc_bh=r["acc_bh"], pot_bh=r["pot_bh"], acc=r["acc"],
            pot=r["pot"], oldacc=r["oldacc"], cost_bh=s["cost_bh"], cost_rel=s["cost_rel"], vel=ic["vel"],
            drift_dt=r["info"]["drift"]["dt"], pos_drift=r["pos_drift"], acc_drift=r["acc_drift"],
            pot_drift=r["pot_drift"], cost_drift=r["info"]["drift"]["cost"], pot_only=rp["pot_only"],
            oldacc_pot=rp["oldacc"])
        print(name, "n=%d cost_bh=%d cost_rel=%d cost_drift=%d" % (ic["pos"].shape[0], s["cost_bh"], s["cost_rel"],
                                                                  r["info"]["drift"]["cost"]))


if __name__ == "__main__":
    main()
