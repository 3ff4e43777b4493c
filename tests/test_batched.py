"""Batched ensembles: CUDA-graph replay of a whole step and the autotuner.

A graph replay must compute exactly what the same uncaptured step computes
(same tree, same OldAcc on the device), and the configuration the autotuner
picks must keep the force error of every system within the bound the default
configuration meets, checked against the FP64 direct sum inside each system.
"""
import numpy as np
import pytest

import ggb200
import ics
import oracle

pytestmark = pytest.mark.gpu


def _ensemble(S=24, nmax=6000, seed=9):
    return ics.ensemble(n_systems=S, nmin=256, nmax=nmax, seed=seed)


def _setup(torch, ic, stream, **kw):
    n = ic["pos"].shape[0]
    rec = ggb200.make_records(ic["pos"], ic["mass"], ic["h"])
    d_rec = torch.from_numpy(rec.view(np.uint8)).cuda()
    t = ggb200.GravityTree(**kw)
    t.set_stream(stream.cuda_stream)
    t.load_device(d_rec, ic["counts"])
    acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    pot = torch.empty(n, dtype=torch.float64, device="cuda")
    t.build()
    t.evaluate_device(acc, pot, err_tol_theta=0.7)
    t.build()
    t.evaluate_device(acc, pot, err_tol_force_acc=0.001)
    return t, d_rec, acc, pot


def test_graph_replay_equals_uncaptured_steps():
    import torch
    ic = _ensemble()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ta, _, acc_a, pot_a = _setup(torch, ic, stream)
        tb, _, acc_b, pot_b = _setup(torch, ic, stream)
        ref = []
        for _ in range(3):                       # uncaptured steps, OldAcc carried on the device
            ta.build()
            ta.evaluate_device(acc_a, pot_a, err_tol_force_acc=0.001)
            ref.append((acc_a.clone(), pot_a.clone()))
        # capture needs every buffer allocated: one uncaptured step first, then restart
        # both contexts from the same state by rerunning the start-up passes
        tb.build()
        tb.evaluate_device(acc_b, pot_b, err_tol_force_acc=0.001)
        tb.build()
        tb.evaluate_device(acc_b, pot_b, err_tol_theta=0.7)
        tb.build()
        tb.evaluate_device(acc_b, pot_b, err_tol_force_acc=0.001)
        tb.capture_step(acc_b, pot_b, err_tol_force_acc=0.001)
        for k in range(3):
            launches0 = ggb200.kernel_launches()
            tb.launch_step()
            assert ggb200.kernel_launches() > launches0
            torch.cuda.synchronize()
            assert torch.equal(acc_b, ref[k][0]) and torch.equal(pot_b, ref[k][1]), "replay %d differs" % k
        sa, sb = ta.last_stats(), tb.last_stats()
        assert sa["interactions"] == sb["interactions"] and sb["error_word"] == 0
        ta.close()
        tb.close()


def test_capture_and_launch_reject_bad_calls():
    t = ggb200.GravityTree()
    with pytest.raises(ggb200.GravityError):
        t.launch_step()                          # nothing captured
    ic = ics.plummer(2000, seed=3)
    t.load(ic["pos"], ic["mass"], ic["h"])
    with pytest.raises(ggb200.GravityError):
        t.capture_step(None)                     # no output buffer
    t.close()


def _per_system_p99(ic, acc, per=24, seed=5):
    rng = np.random.default_rng(seed)
    off = np.concatenate([[0], np.cumsum(ic["counts"])])
    worst = 0.0
    for s, n in enumerate(ic["counts"]):
        o, n = int(off[s]), int(n)
        tg = np.sort(rng.choice(n, min(per, n), replace=False)).astype(np.int32)
        a_dir = oracle.direct_sum(ic["pos"][o:o + n], ic["mass"][o:o + n], ic["h"][o:o + n], targets=tg)[0]
        _, p99, _ = ics.error_stats(acc[o + tg], a_dir)
        worst = max(worst, p99)
    return worst


def test_autotune_keeps_the_force_error_and_returns_a_valid_config():
    import torch
    ic = _ensemble(S=16, nmax=4000, seed=11)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        t, _, acc, pot = _setup(torch, ic, stream)
        t.build()
        t.evaluate_device(acc, pot, err_tol_force_acc=0.001)
        torch.cuda.synchronize()
        base = _per_system_p99(ic, acc.cpu().numpy())
        cfg, ms = t.autotune(err_tol_force_acc=0.001)
        assert cfg["leaf_size"] in (8, 16) and cfg["group_size"] in (32, 64)
        assert cfg["flush"] in (64, 128) and cfg["blocks_per_sm"] in (2, 3) and ms > 0
        t.build()
        t.evaluate_device(acc, pot, err_tol_force_acc=0.001)
        torch.cuda.synchronize()
        assert t.last_stats()["error_word"] == 0
        tuned = _per_system_p99(ic, acc.cpu().numpy())
        # the accuracy gate holds every system to 1.1x the base configuration
        # on its own sample; on this independent sample allow sampling noise
        assert tuned < 2e-3 and tuned <= 1.25 * base + 1e-5
        t.close()


def test_tuner_gate_refuses_a_less_accurate_configuration():
    """Leaf buckets of 16 on the reference's clustered golden put the potential
    energy further from the direct sum than the reference tree does (and than
    the default leaf 8): the autotuner's gate refuses it, while configurations
    that change no opening decision (flush threshold, blocks per SM, node
    staging) pass."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "clustered_1500.npz"))
    tol = float(g["tol"])
    with ggb200.GravityTree() as t:
        t.load(g["pos"], g["mass"], g["h"])
        t.build()
        a1, _, _, _ = t.evaluate(err_tol_theta=0.7)
        t.evaluate(old_acc=np.linalg.norm(a1, axis=1), err_tol_force_acc=tol)
        assert not t.tune_accuracy(err_tol_force_acc=tol, leaf_size=16)
        assert t.tune_accuracy(err_tol_force_acc=tol, flush=64)
        assert t.tune_accuracy(err_tol_force_acc=tol, blocks_per_sm=3, node_staging=1)
        # the context is left as it was: the same walk gives the same bits
        a2, p2, _, _ = t.evaluate(old_acc=np.linalg.norm(a1, axis=1), err_tol_force_acc=tol)
        a3, p3, _, _ = t.evaluate(old_acc=np.linalg.norm(a1, axis=1), err_tol_force_acc=tol)
        assert np.array_equal(a2, a3) and np.array_equal(p2, p3)


def test_split_system_step_on_one_gpu_equals_plain_evaluation():
    """multi.SplitSystem at world size 1 (the gather is the identity): the
    own-range walk through an active list equals the plain walk."""
    import torch
    import multi
    ic = ics.galaxy(n_halo=14000, n_disk=6000, seed=13)
    n = ic["pos"].shape[0]
    rec = torch.from_numpy(ggb200.make_records(ic["pos"], ic["mass"], ic["h"]).view(np.uint8)).cuda()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ta = ggb200.GravityTree()
        ta.set_stream(stream.cuda_stream)
        split = multi.SplitSystem(None, ta, torch, "cuda")
        acc_a = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        pot_a = torch.empty(n, dtype=torch.float64, device="cuda")
        split.step(rec, acc_a, pot_a, err_tol_theta=0.7)
        split.step(rec, acc_a, pot_a, err_tol_force_acc=0.001)
        tb = ggb200.GravityTree()
        tb.set_stream(stream.cuda_stream)
        acc_b = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        pot_b = torch.empty(n, dtype=torch.float64, device="cuda")
        tb.load_device(rec, [n])
        tb.build()
        tb.evaluate_device(acc_b, pot_b, err_tol_theta=0.7)
        tb.build()
        tb.evaluate_device(acc_b, pot_b, err_tol_force_acc=0.001)
        torch.cuda.synchronize()
        assert torch.equal(acc_a, acc_b) and torch.equal(pot_a, pot_b)
        ta.close()
        tb.close()


def test_autotune_for_an_active_subset():
    """The search on the walk of a 10% active subset (individual timesteps):
    a valid configuration, and the subset's forces with it stay within the
    default configuration's error against the FP64 direct sum."""
    import torch
    ic = ics.clustered(200000, seed=17, n_clumps=40)
    n = ic["pos"].shape[0]
    act = ics.random_active(n, 0.1, seed=18).astype(np.int32)
    tg = act[:: 16]
    acc_d, _ = oracle.direct_sum(ic["pos"], ic["mass"], ic["h"], targets=tg)
    rows = np.searchsorted(act, tg)
    with ggb200.GravityTree() as t:
        t.load(ic["pos"], ic["mass"], ic["h"])
        t.build()
        a1, _, _, _ = t.evaluate(err_tol_theta=0.7)
        old = np.linalg.norm(a1, axis=1)
        base, _, _, _ = t.evaluate(active=act, old_acc=old, err_tol_force_acc=0.001)
        d_act = torch.from_numpy(act).cuda()
        cfg, ms = t.autotune(err_tol_force_acc=0.001, d_active=d_act, n_active=act.size)
        assert cfg["leaf_size"] in (8, 16) and cfg["group_size"] in (32, 64) and ms > 0
        t.build()
        tuned, _, _, st = t.evaluate(active=act, old_acc=old, err_tol_force_acc=0.001)
    assert st["error_word"] == 0
    b50, b99, _ = ics.error_stats(base[rows], acc_d)
    t50, t99, _ = ics.error_stats(tuned[rows], acc_d)
    assert t99 <= 1.25 * b99 + 1e-5, (t99, b99)


def test_two_part_graph_equals_uncaptured_steps_and_stale_graph_is_refused():
    """The step captured as two graphs (build, walk) and replayed gives the
    bits of the same steps issued launch by launch; after a buffer of the
    context grows (a larger system set), the stale graphs are refused."""
    import torch
    ic = ics.clustered(120000, seed=95, n_clumps=20)
    n = ic["pos"].shape[0]
    rec = torch.from_numpy(ggb200.make_records(ic["pos"], ic["mass"], ic["h"]).view(np.uint8)).cuda()
    res = []
    for graphs in (False, True):
        stream = torch.cuda.Stream()
        with ggb200.GravityTree(group_size=64) as t:
            t.set_stream(stream.cuda_stream)
            t.load_device(rec, [n])
            d_acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
            d_pot = torch.empty(n, dtype=torch.float64, device="cuda")
            t.build()
            t.evaluate_device(d_acc, d_pot, err_tol_theta=0.7)
            t.build()
            t.evaluate_device(d_acc, d_pot, err_tol_force_acc=0.001)
            if graphs:
                t.capture_step_parts(d_acc, d_pot, err_tol_force_acc=0.001)
            for _ in range(3):
                if graphs:
                    t.launch_step_part(0)
                    t.launch_step_part(1)
                else:
                    t.build()
                    t.evaluate_device(d_acc, d_pot, err_tol_force_acc=0.001)
            stream.synchronize()
            res.append((d_acc.cpu().numpy(), d_pot.cpu().numpy(), t.last_stats()["interactions"]))
            if graphs:
                big = torch.cat([rec, rec])
                t.load_device(big, [n, n])
                t.build()
                with pytest.raises(ggb200.GravityError):
                    t.launch_step_part(1)
    (a0, p0, i0), (a1, p1, i1) = res
    assert np.array_equal(a0, a1) and np.array_equal(p0, p1) and i0 == i1
