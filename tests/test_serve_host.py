"""Host logic of the serving loop on CPU, with a stand-in for the library context.

The stand-in keeps each system's positions, drifts them like the device
tree, finishes its work after a seeded random number of polls (so batches
complete out of order) and returns a result that depends only on the
system's own current positions.  The scheduler must then give every request
the result it gets alone, respect the memory budget, evict and re-solve
evicted systems at their drifted positions, and never drift a system twice
in one launch.
"""
import numpy as np
import pytest

import serve


class FakeTree:
    polls_rng = np.random.default_rng(7)
    bytes_per_particle = 600
    fixed = 64 << 20

    def __init__(self, **cfg):
        self.cfg = cfg
        self.n = 0
        self.closed = False

    def load_systems(self, systems):
        self.pos = np.concatenate([s["pos"] for s in systems]).copy()
        self.vel = np.concatenate([s["vel"] for s in systems])
        self.counts = np.array([s["pos"].shape[0] for s in systems])
        self.off = np.concatenate([[0], np.cumsum(self.counts)])
        self.n = int(self.counts.sum())
        self.cap = max(getattr(self, "cap", 0), self.n)
        self.built = False
        self.drifts = []

    def build(self):
        self.built = True

    def drift(self, dts):
        assert self.built
        dts = np.asarray(dts)
        assert dts.shape == (len(self.counts),)
        for s, dt in enumerate(dts):
            lo, hi = self.off[s], self.off[s + 1]
            self.pos[lo:hi] = self.pos[lo:hi] + self.vel[lo:hi] * dt
        self.drifts.append(dts.copy())

    def evaluate_async(self, active=None, err_tol_force_acc=0.0, err_tol_theta=0.0, copy_acc=True, copy_pot=True):
        assert self.built
        idx = np.arange(self.n) if active is None else np.asarray(active)
        sys_of = np.searchsorted(self.off, idx, side="right") - 1
        # a result that depends on the particle's own system only
        cent = np.array([self.pos[self.off[s]:self.off[s + 1]].mean(axis=0) for s in range(len(self.counts))])
        self.result = (self.pos[idx] - cent[sys_of], np.full(idx.size, float(self.counts.size > 0)) * sys_of * 0)
        self.left = int(self.polls_rng.integers(1, 5))

    def evaluate_async_pinned(self, acc, pot, active=None, err_tol_force_acc=0.0, err_tol_theta=0.0):
        self.evaluate_async(active, err_tol_force_acc, err_tol_theta)
        self.out = (acc, pot)

    def query(self):
        self.left -= 1
        return self.left <= 0

    def fetch(self):
        acc, pot = self.result
        if getattr(self, "out", None) is not None:
            a, p = self.out
            self.out = None
            a[:] = acc
            p[:] = pot + 1.0
            return a, p, {"error_word": 0}
        return acc.copy(), pot.copy() + 1.0, {"error_word": 0}

    def device_bytes(self):
        return self.fixed + self.bytes_per_particle * self.cap

    def close(self):
        self.closed = True


def _pool(k=9, seed=11):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        n = int(rng.integers(50, 3000))
        out.append({"pos": rng.normal(size=(n, 3)), "vel": rng.normal(size=(n, 3)), "mass": np.full(n, 1.0 / n),
                    "h": np.full(n, 0.01)})
    return out


def _expected(reqs):
    """Each request's result computed directly from its own system."""
    drift = {}
    out = {}
    for r in reqs:
        sid = r.rid if r.kind == "new" else r.target
        s = r.system if r.kind == "new" else next(q.system for q in reqs if q.rid == sid)
        drift[sid] = drift.get(sid, 0.0) + (r.dt if r.kind == "reeval" else 0.0)
        pos = s["pos"] + s["vel"] * drift[sid] if drift[sid] else s["pos"]
        out[r.rid] = pos - pos.mean(axis=0)
    return out


@pytest.mark.parametrize("batching", [True, False])
def test_every_request_gets_its_own_result(batching):
    pool = _pool()
    reqs = serve.make_trace(pool, rate=1e6, window_s=3e-4, frac_reeval=0.4, dt=1e-2, recent=5, seed=3)[:80]
    srv = serve.Server(batching=batching, max_batch_particles=6000, max_inflight=3, tree_factory=FakeTree,
                       pinned_results=batching, result_alloc=np.empty)
    serve.run_trace(srv, reqs, realtime=False)
    exp = _expected(reqs)
    for r in reqs:
        assert r.acc is not None and r.acc.shape == exp[r.rid].shape
        # one drift per system and launch: the fake drifts positions with separate roundings
        assert np.allclose(r.acc, exp[r.rid], rtol=0, atol=1e-12), r.rid
    if batching:
        assert srv.n_batches < len(reqs)
    else:
        assert srv.n_batches == len(reqs)
    for c in srv.contexts:
        for d in c.tree.drifts:
            assert np.count_nonzero(d) >= 1
    srv.close()


def test_budget_is_respected_and_misses_are_resolved():
    pool = _pool(k=12, seed=12)
    budget = 3 * (FakeTree.fixed + FakeTree.bytes_per_particle * 6000)
    srv = serve.Server(budget_bytes=budget, batching=True, max_batch_particles=6000, max_inflight=2,
                       tree_factory=FakeTree, result_alloc=np.empty)
    first = [serve.Request(i, "new", 0.0, system=pool[i]) for i in range(12)]
    serve.run_trace(srv, first, realtime=False)
    # the earliest systems were evicted to make room: their re-evaluations miss
    later = [serve.Request(12 + k, "reeval", 0.0, target=k % 3, dt=1e-2) for k in range(6)]
    later += [serve.Request(18, "reeval", 0.0, target=11, dt=1e-2)]
    serve.run_trace(srv, later, realtime=False)
    assert srv.evictions > 0
    assert all(r.miss for r in later[:3]) and not later[-1].miss
    assert srv.peak_bytes <= budget
    exp = _expected(first + later)
    for r in first + later:
        assert np.allclose(r.acc, exp[r.rid], rtol=0, atol=1e-12), (r.rid, r.miss)
    srv.close()


def test_request_larger_than_the_budget_is_refused():
    pool = _pool(k=1, seed=13)
    reqs = [serve.Request(0, "new", 0.0, system=pool[0])]
    srv = serve.Server(budget_bytes=1e6, tree_factory=FakeTree, result_alloc=np.empty)
    with pytest.raises(MemoryError):
        serve.run_trace(srv, reqs, realtime=False)


def test_trace_is_poisson_with_the_requested_mix():
    pool = _pool(k=4, seed=14)
    reqs = serve.make_trace(pool, rate=2000.0, window_s=3.0, frac_reeval=0.3, seed=5)
    t = np.array([r.arrival for r in reqs])
    assert 5400 < len(reqs) < 6600 and np.all(np.diff(t) > 0) and t[-1] <= 3.0
    frac = np.mean([r.kind == "reeval" for r in reqs])
    assert 0.27 < frac < 0.33
    news = {r.rid for r in reqs if r.kind == "new"}
    assert all(r.target in news and r.target < r.rid for r in reqs if r.kind == "reeval")
