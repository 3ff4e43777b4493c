"""Node records staged by the bulk-copy (TMA) engine against per-lane cp.async.

The walk copies the next round's node records into shared memory either lane
by lane (cp.async) or as one bulk copy per run of consecutive records,
completing on an mbarrier.  The records are the same bytes either way, so
forces, potentials and interaction counts must be bitwise equal: one system
and many, all targets or a subset.  (The exact and potential-only walks stage
per lane in both settings; the last case and the potentials check that the
setting leaves them alone.)
"""
import numpy as np
import pytest

import ggb200
import ics

pytestmark = pytest.mark.gpu


def _walks(ic, staging, active=None, group_size=32):
    import torch
    n = ic["pos"].shape[0]
    stream = torch.cuda.Stream()
    rec = torch.from_numpy(ggb200.make_records(ic["pos"], ic["mass"], ic["h"]).view(np.uint8)).cuda()
    t = ggb200.GravityTree(node_staging=staging, group_size=group_size)
    t.set_stream(stream.cuda_stream)
    t.load_device(rec, ic["counts"])
    acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    pot = torch.empty(n, dtype=torch.float64, device="cuda")
    nint = torch.empty(n, dtype=torch.int32, device="cuda")
    d_act, n_act = None, 0
    if active is not None:
        d_act = torch.from_numpy(active.astype(np.int32)).cuda()
        n_act = active.size
    t.build()
    t.evaluate_device(acc, pot, err_tol_theta=0.7)
    out = []
    for _ in range(2):
        t.build()
        t.evaluate_device(acc, pot, d_active=d_act, n_active=n_act, err_tol_force_acc=0.001, d_ninter=nint)
        stream.synchronize()
        out += [acc.cpu().numpy().copy(), pot.cpu().numpy().copy(), nint.cpu().numpy().copy()]
    t.evaluate_potential_device(pot)
    stream.synchronize()
    out.append(pot.cpu().numpy().copy())
    st = t.last_stats()
    t.close()
    return out, st


@pytest.mark.parametrize("case", ["galaxy", "ensemble", "subset", "exact"])
def test_bulk_copy_staging_equals_per_lane_staging(case):
    active, gs = None, 32
    if case == "galaxy":
        ic = ics.galaxy(50000, 20000, seed=91)
        ic["counts"] = [ic["pos"].shape[0]]
    elif case == "ensemble":
        ic = ics.ensemble(n_systems=10, nmin=256, nmax=8000, seed=92)
    elif case == "subset":
        ic = ics.clustered(60000, seed=93, n_clumps=40)
        ic["counts"] = [ic["pos"].shape[0]]
        active = ics.random_active(60000, 0.15, seed=94)
    else:
        ic = ics.plummer(3000, seed=95)
        ic["counts"] = [ic["pos"].shape[0]]
        gs = 1
    a, sa = _walks(ic, 0, active, gs)
    b, sb = _walks(ic, 1, active, gs)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert sa["interactions"] == sb["interactions"] and sa["nodes_tested"] == sb["nodes_tested"]
    assert sb["error_word"] == 0
