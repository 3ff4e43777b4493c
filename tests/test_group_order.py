"""Walk groups handed out by measured cost.

Each walk records per target its group's device cycles per target; the next
walk of the context hands its groups out most expensive first.  Only the time
at which a group runs changes: forces, potentials, interaction counts and
OldAcc must be bitwise equal to the walk that hands groups out in target
order, for full and active-subset walks, one system or many, and for the
potential-only walk.
"""
import numpy as np
import pytest

import ggb200
import ics

pytestmark = pytest.mark.gpu


def _steps(ic, group_order, active=None, potential=False):
    import torch
    n = ic["pos"].shape[0]
    stream = torch.cuda.Stream()
    rec = torch.from_numpy(ggb200.make_records(ic["pos"], ic["mass"], ic["h"]).view(np.uint8)).cuda()
    t = ggb200.GravityTree(group_order=group_order)
    t.set_stream(stream.cuda_stream)
    t.load_device(rec, ic["counts"])
    acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    pot = torch.empty(n, dtype=torch.float64, device="cuda")
    nint = torch.empty(n, dtype=torch.int32, device="cuda")
    t.build()
    t.evaluate_device(acc, pot, err_tol_theta=0.7)
    d_act, n_act = None, 0
    if active is not None:
        d_act = torch.from_numpy(active.astype(np.int32)).cuda()
        n_act = active.size
    out = []
    for _ in range(3):   # from the second relative walk on, groups run in cost order
        t.build()
        t.evaluate_device(acc, pot, d_active=d_act, n_active=n_act, err_tol_force_acc=0.001, d_ninter=nint)
        stream.synchronize()
        m = n if active is None else n_act   # a subset walk writes its first n_act slots only
        out.append((acc[:m].cpu().numpy().copy(), pot[:m].cpu().numpy().copy(), nint[:m].cpu().numpy().copy()))
    if potential:
        t.evaluate_potential_device(pot)
        stream.synchronize()
        out.append((None, pot.cpu().numpy().copy(), None))
    st = t.last_stats()
    t.close()
    return out, st


def _same(a, b):
    for (xa, pa, na), (xb, pb, nb) in zip(a, b):
        if xa is not None:
            assert np.array_equal(xa, xb)
            assert np.array_equal(na, nb)
        assert np.array_equal(pa, pb)


@pytest.mark.parametrize("case", ["galaxy", "ensemble"])
def test_cost_order_changes_no_result(case):
    if case == "galaxy":
        ic = ics.galaxy(60000, 20000, seed=77)
        ic["counts"] = [ic["pos"].shape[0]]
    else:
        ic = ics.ensemble(n_systems=12, nmin=256, nmax=9000, seed=78)
    a, sa = _steps(ic, 1, potential=True)
    b, sb = _steps(ic, 0, potential=True)
    _same(a, b)
    assert sa["interactions"] == sb["interactions"] and sa["nodes_tested"] == sb["nodes_tested"]


def test_cost_order_with_active_subset():
    ic = ics.plummer(40000, seed=79)
    ic["counts"] = [ic["pos"].shape[0]]
    active = ics.random_active(40000, 0.2, seed=80)
    a, _ = _steps(ic, 1, active=active)
    b, _ = _steps(ic, 0, active=active)
    _same(a, b)
