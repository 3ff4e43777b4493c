"""The serving loop: continuous batching, resident trees, memory admission.

Each result must be the same whether its request is served alone or mixed
with others (batched into shared contexts, overlapping on the device):
systems never interact, so the results are required to be bitwise equal.
With a small memory budget, evicted systems are solved again at their drifted
positions and must stay within the force-error bound of the direct sum.
"""
import numpy as np
import pytest

import ics
import oracle
import serve

pytestmark = pytest.mark.gpu


def _pool(k=10, seed=501):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(800), np.log(30000), k)).astype(int)
    return [ics.serving_system(i % 3, int(n), seed + i) for i, n in enumerate(sizes)]


def _trace(pool, n=48, seed=502):
    reqs = serve.make_trace(pool, rate=1e6, window_s=3e-4, frac_reeval=0.35, dt=1e-3, recent=6, seed=seed)
    return reqs[:n]


def _alone(reqs):
    """Serve each system's requests (its new solve, then its re-evaluations in
    order) in a server of its own, one request at a time."""
    out = {}
    by_sys = {}
    for r in reqs:
        by_sys.setdefault(r.rid if r.kind == "new" else r.target, []).append(r)
    for sid, rs in by_sys.items():
        srv = serve.Server(batching=False)
        copies = [serve.Request(r.rid, r.kind, 0.0, system=r.system, target=r.target, dt=r.dt) for r in rs]
        serve.run_trace(srv, copies, realtime=False)
        for c in copies:
            out[c.rid] = c
        srv.close()
    return out


def test_results_same_alone_and_in_the_mix():
    pool = _pool()
    reqs = _trace(pool)
    assert any(r.kind == "reeval" for r in reqs) and any(r.kind == "new" for r in reqs)
    srv = serve.Server(batching=True, max_batch_particles=60000, max_inflight=4)
    serve.run_trace(srv, reqs, realtime=False)
    assert srv.n_batches < len(reqs)            # requests were batched
    assert max(len(items) for items in _batch_sizes(reqs).values()) > 1
    alone = _alone(reqs)
    for r in reqs:
        a = alone[r.rid]
        assert not r.miss and not a.miss
        assert np.array_equal(r.acc, a.acc) and np.array_equal(r.pot, a.pot), (r.rid, r.kind)
    srv.close()


def _batch_sizes(reqs):
    b = {}
    for r in reqs:
        b.setdefault(r.batch, []).append(r)
    return b


def test_reevaluation_follows_the_drift():
    pool = _pool(k=3, seed=503)
    reqs = [serve.Request(0, "new", 0.0, system=pool[0]),
            serve.Request(1, "reeval", 0.0, target=0, dt=2e-3),
            serve.Request(2, "reeval", 0.0, target=0, dt=2e-3)]
    srv = serve.Server()
    serve.run_trace(srv, reqs, realtime=False)
    s = pool[0]
    moved = s["pos"] + s["vel"] * 2e-3
    moved = moved + s["vel"] * 2e-3
    acc_d, _ = oracle.direct_sum(moved, s["mass"], s["h"])
    assert ics.error_stats(reqs[2].acc, acc_d)[1] < 2e-3
    acc_0, _ = oracle.direct_sum(s["pos"], s["mass"], s["h"])
    assert ics.error_stats(reqs[0].acc, acc_0)[1] < 2e-3
    srv.close()


def test_small_budget_evicts_and_solves_misses_afresh():
    pool = _pool(k=8, seed=504)
    reqs = _trace(pool, n=40, seed=505)
    srv = serve.Server(budget_bytes=700e6, max_batch_particles=40000, max_inflight=3)
    serve.run_trace(srv, reqs, realtime=False)
    assert srv.evictions > 0
    assert srv.peak_bytes <= srv.budget
    assert all(r.acc is not None for r in reqs)
    misses = [r for r in reqs if r.miss]
    for r in misses[:4]:
        s = r.system
        # drift accumulated by this system's re-evaluations up to this one
        d = sum(q.dt for q in reqs if q.kind == "reeval" and q.target == r.target and q.rid <= r.rid)
        moved = s["pos"] + s["vel"] * d
        acc_d, _ = oracle.direct_sum(moved, s["mass"], s["h"])
        assert ics.error_stats(r.acc, acc_d)[1] < 2e-3
    srv.close()


def test_device_pool_reservation():
    import ggb200
    ggb200.reserve_device_pool(1 << 30)      # maps 1 GB into this process's pool once
    ggb200.reserve_device_pool(1 << 30)      # served from the pool the second time
    with pytest.raises(ggb200.GravityError):
        ggb200.reserve_device_pool(-1)


def test_pinned_results_equal_the_copied_ones():
    """gg_evaluate_async_pinned writes the same bits into the caller's
    page-locked arrays as gg_evaluate_async + gg_fetch_results copy out (two
    contexts taken through the same steps), for all targets and then an active
    subset; a pageable array is refused; gg_host_free refuses a pointer that
    is not one of its blocks."""
    import ctypes
    import ggb200
    sysd = ics.serving_system(0, 20000, 601)
    act = np.sort(np.random.default_rng(602).choice(20000, 3000, replace=False)).astype(np.int32)
    res = []
    for pinned in (False, True):
        with ggb200.GravityTree() as t:
            t.load_systems([sysd])
            t.build()
            t.evaluate_async(err_tol_theta=0.7, copy_acc=False, copy_pot=False)
            t.fetch()
            out = []
            for active in (None, act):
                n = 20000 if active is None else act.size
                if pinned:
                    acc, pot = ggb200.host_empty((n, 3)), ggb200.host_empty(n)
                    t.evaluate_async_pinned(acc, pot, active=active, err_tol_force_acc=0.001)
                    a, p, st = t.fetch()
                    assert a is acc and p is pot
                else:
                    t.evaluate_async(active=active, err_tol_force_acc=0.001)
                    a, p, st = t.fetch()
                assert st["n_targets"] == n
                out.append((a, p, st["interactions"]))
            if pinned:
                with pytest.raises(ggb200.GravityError):
                    t.evaluate_async_pinned(np.empty((20000, 3)), None, err_tol_force_acc=0.001)
            res.append(out)
    for (a0, p0, i0), (a1, p1, i1) in zip(*res):
        assert np.array_equal(a0, a1) and np.array_equal(p0, p1) and i0 == i1
    assert ggb200.load_library().gg_host_free(ctypes.c_void_p(0x1000)) == -1
