"""GIZMO itself driving the B200 library through its C host code.

oracle/_ref/gizmo_b200 is the reference code (begrun, domain decomposition,
the two start-up gravity passes of compute_grav_accelerations) with the
reference's own gravity/gravtree.c patched by oracle/patch_gravtree.py with
the GRAVITY_GPU_B200 blocks that INTEGRATION.md documents: inside
gravity_tree(), force_treebuild becomes gravtree_b200_build() and the walk /
export loop becomes gravtree_b200_walk() (gizmo-public_b200/host/
gravtree_b200.c, which hands GIZMO's own P[] records, strided, to the C ABI).
Everything else is the reference's: move_particles and
rearrange_particle_sequence before a build, and the post-processing that
multiplies by G, sets OldAcc = |a|/G and switches to the relative criterion.
The same inputs go through the plain reference binary; results must agree to
the tree's accuracy.  After the start-up passes, both binaries also
re-evaluate the system a drift later without rebuilding the tree: the
reference drifts its nodes inside the walk (force_drift_node); the host code
drifts the device tree's nodes (gg_drift) and hands it P[].Pos
(gg_set_positions).
"""
import numpy as np
import pytest

import ics
import oracle
import ref_runner

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not ref_runner.available(ref_runner.BIN_B200) or not ref_runner.available(),
                    reason="reference binaries not built (oracle/build_ref.sh needs the reference tree)")
@pytest.mark.parametrize("model", ["plummer", "galaxy"])
def test_gizmo_with_b200_gravity_matches_reference(model):
    if model == "plummer":
        ic = ics.plummer(8192, seed=201)
    else:
        ic = ics.galaxy(n_halo=6000, n_disk=2192, seed=202)
    ref = ref_runner.run(ic, threads=4, drift_dt=0.002)
    gpu = ref_runner.run(ic, threads=4, binary=ref_runner.BIN_B200, drift_dt=0.002)
    acc_d, pot_d = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"])
    r50, r99, _ = ics.error_stats(ref["acc"], acc_d)
    g50, g99, _ = ics.error_stats(gpu["acc"], acc_d)
    assert g50 <= 1.1 * r50 and g99 <= 1.1 * r99, (g50, g99, r50, r99)
    # OldAcc = |a|/G written back into P[] by the host code (G = 1 here)
    assert np.allclose(gpu["oldacc"], np.linalg.norm(gpu["acc"], axis=1), rtol=1e-12)
    assert np.allclose(gpu["pot"], pot_d, rtol=2e-3)
    assert gpu["info"]["startup"]["cost_rel"] > 0
    # the re-evaluation after the drift, against the direct sum at the drifted positions
    assert gpu["info"]["drift"]["dt"] == ref["info"]["drift"]["dt"]
    assert np.array_equal(gpu["pos_drift"], ref["pos_drift"])   # GIZMO's own particle drift in both
    acc_dd, _ = oracle.direct_sum(ref["pos_drift"], ic["mass"], ic["h"])
    r50, r99, _ = ics.error_stats(ref["acc_drift"], acc_dd)
    g50, g99, _ = ics.error_stats(gpu["acc_drift"], acc_dd)
    assert g50 <= 1.1 * r50 and g99 <= 1.1 * r99, (g50, g99, r50, r99)


@pytest.mark.skipif(not ref_runner.available(ref_runner.BIN_B200),
                    reason="reference binaries not built (oracle/build_ref.sh needs the reference tree)")
@pytest.mark.parametrize("model", ["plummer", "galaxy"])
def test_gizmo_peano_hilbert_order_on_the_gpu(model, monkeypatch):
    """peano_hilbert_order_b200() inside GIZMO: after a shuffle of P[] it
    restores GIZMO's own order down to 21-bit cells (the harness compares the
    key prefixes along both orders with GIZMO's own key function)."""
    ic = ics.plummer(20000, seed=211) if model == "plummer" else ics.galaxy(n_halo=12000, n_disk=8000, seed=212)
    monkeypatch.setenv("GG_CHECK_PH_ORDER", "1")
    r = ref_runner.run(ic, threads=4, binary=ref_runner.BIN_B200)
    ph = r["info"]["phorder"]
    assert ph["n"] == ic["pos"].shape[0] and ph["moved"] > ph["n"] // 2
    assert ph["key21_sorted"] == 1 and ph["same_as_reference"] == 1
