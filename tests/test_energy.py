"""FP64 energy and momentum checks on the device (gg_energy_device).

W = 1/2 sum m phi (the potential energy of global.c:54) and sum m a per
system, checked against the same sums formed on the host from the outputs,
and, for exact forces (the FP64 direct sum), the momentum sum vanishing.
"""
import numpy as np
import pytest

import ggb200
import ics

pytestmark = pytest.mark.gpu


def test_energy_and_momentum_sums_per_system():
    import torch
    a = ics.plummer(6000, seed=401)
    b = ics.galaxy(n_halo=3000, n_disk=1000, seed=402)
    b["pos"] = b["pos"] + 50.0
    pos = np.concatenate([a["pos"], b["pos"]])
    mass = np.concatenate([a["mass"], b["mass"]])
    h = np.concatenate([a["h"], b["h"]])
    counts = [6000, 4000]
    with ggb200.GravityTree() as t:
        t.load(pos, mass, h, counts=counts)
        t.build()
        a1, _, _, _ = t.evaluate(err_tol_theta=0.7)
        acc, pot, _, _ = t.evaluate(old_acc=np.linalg.norm(a1, axis=1), err_tol_force_acc=0.001)
        d_acc = torch.from_numpy(acc).cuda()
        d_pot = torch.from_numpy(pot).cuda()
        e = t.energy_device(d_acc, d_pot)
        e_pot_only = t.energy_device(None, d_pot)
    m32 = mass.astype(np.float32).astype(np.float64)   # masses are stored in FP32
    off = [0, 6000, 10000]
    for s in range(2):
        sl = slice(off[s], off[s + 1])
        W = 0.5 * np.sum(m32[sl] * pot[sl])
        F = (m32[sl, None] * acc[sl]).sum(axis=0)
        assert abs(e[s, 0] - W) <= 1e-12 * abs(W)
        assert np.allclose(e[s, 1:], F, rtol=1e-10, atol=1e-13)
        assert e_pot_only[s, 0] == e[s, 0] and np.all(e_pot_only[s, 1:] == 0)
        # the tree's momentum residual is small next to the typical force
        scale = np.sum(m32[sl] * np.linalg.norm(acc[sl], axis=1))
        assert np.linalg.norm(e[s, 1:]) < 1e-2 * scale


def test_direct_forces_conserve_momentum():
    import torch
    ic = ics.plummer(3000, seed=403)
    n = 3000
    dp, dm, dh = (torch.from_numpy(x).cuda() for x in (ic["pos"], ic["mass"], ic["h"]))
    dacc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    dpot = torch.empty(n, dtype=torch.float64, device="cuda")
    tg = torch.arange(n, dtype=torch.int32, device="cuda")
    ggb200.direct_sum_fp64(dp, dm, dh, n, tg, n, dacc, dpot)
    torch.cuda.synchronize()
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.build()
        e = t.energy_device(dacc, dpot)
    scale = np.sum(ic["mass"] * np.linalg.norm(dacc.cpu().numpy(), axis=1))
    assert np.linalg.norm(e[0, 1:]) < 1e-7 * scale   # pairwise forces cancel (FP32 masses aside)
