"""Serving loop: force-evaluation solves on one GPU with continuous batching.

Requests arrive over time.  A request is either
  - a new system (positions, velocities, masses, kernel radii): GIZMO's
    start-up evaluation of it (accel.c:47-50) -- tree build, Barnes-Hut pass
    for OldAcc, relative-criterion pass -- or
  - a re-evaluation of a resident system after a drift by dt: the system's
    tree stays on the device and is drifted (force_drift_node,
    gravity/forcetree_update.c:265-338) and walked again with the OldAcc of
    its previous evaluation, without a rebuild.

Continuous batching: new systems that are waiting when a slot frees up are
loaded together into one library context (one set of launches for all of
them) and overlap on the device with the batches and re-evaluations already
running, each context on its own CUDA stream.  Re-evaluations of systems that
share a context are drifted and walked together.  Admission is against a
device-memory budget: a batch is admitted only when the memory the contexts
hold (counted by gg_device_bytes) plus its predicted need fits; otherwise
the least recently used idle contexts are evicted (their systems stop being
resident) or the batch waits.  A re-evaluation whose system was evicted is
served as a new solve of the drifted system (a "miss").

The plain form (batching=False) serves one request at a time, one system per
launch sequence, with the same library calls.

Finished launches are fetched (results copied out of the library's pinned
buffers by all host threads) by the scheduler itself; threaded=True hands the
fetches to a completion thread instead.  With pinned_results=True the relative
pass copies its results straight into page-locked arrays allocated for that
launch (ggb200.host_empty, from the library's host cache) and each request's
results are views of them, so a finished launch costs the scheduler no host
copy.  That pays only where requests' results are released as they are
consumed, so that the blocks go back to the cache: a caller that keeps every
result makes each launch page-lock fresh memory, which costs far more than
the copy (the 2,000 req/s benchmark trace, which keeps all results, ran 4x
slower so).

The latency of a request is from its arrival to its result in host memory.
"""
import collections
import queue
import threading
import time

import numpy as np

import ggb200

STARTUP_THETA = 0.7   # GIZMO's start-up Barnes-Hut opening angle (begrun.c:2368)


class Request:
    """One solve.  kind "new": `system` holds pos, vel, mass, h; kind
    "reeval": `target` is the request id of the system to drift by `dt`."""
    __slots__ = ("rid", "kind", "arrival", "system", "target", "dt", "n", "t_done", "acc", "pot", "miss", "batch")

    def __init__(self, rid, kind, arrival, system=None, target=None, dt=0.0):
        self.rid, self.kind, self.arrival = rid, kind, arrival
        self.system, self.target, self.dt = system, target, dt
        self.n = 0 if system is None else int(system["pos"].shape[0])
        self.t_done = None
        self.acc = self.pot = None
        self.miss = False
        self.batch = -1


class _Context:
    """A library context holding the trees of one admitted batch of systems."""

    def __init__(self, tree):
        self.tree = tree
        self.sids = []            # system ids (request ids of their new solves), in load order
        self.offsets = None       # particle offsets of the systems
        self.busy = False
        self.last_use = 0.0
        self.bytes = 0

    def range_of(self, k):
        return int(self.offsets[k]), int(self.offsets[k + 1])


class Server:
    def __init__(self, budget_bytes=120e9, tol=0.001, batching=True, max_batch_particles=8 << 20,
                 max_batch_systems=1024, max_inflight=16, leaf=8, group=32, flush=128, device=0, tree_factory=None,
                 threaded=False, reserve=False, pinned_results=False, result_alloc=None):
        self.budget = float(budget_bytes)
        self.tol = tol
        self.batching = batching
        self.max_batch_particles = int(max_batch_particles) if batching else 1
        self.max_batch_systems = int(max_batch_systems) if batching else 1
        self.max_inflight = int(max_inflight) if batching else 1
        self.cfg = dict(leaf_size=leaf, group_size=group, flush=flush, device=device)
        self.tree_factory = tree_factory or ggb200.GravityTree
        self.pinned_results = pinned_results
        self.result_alloc = result_alloc or ggb200.host_empty   # page-locked result arrays (pinned_results)
        if reserve:
            # map the whole budget once, before the first request; a device
            # smaller than the budget keeps what it could map, and admission
            # against the budget still holds
            try:
                ggb200.reserve_device_pool(self.budget, device)
            except ggb200.GravityError as e:
                if e.status != -3:   # GG_ERR_NOMEM
                    raise
        self.pending_new = collections.deque()
        self.pending_re = collections.deque()
        self.resident = {}           # system id -> (_Context, index in context)
        self.systems = {}            # system id -> host arrays (for a rebuild after eviction)
        self.drifted = {}            # system id -> accumulated drift time
        self.unsolved = set()        # systems whose (re-)solve is waiting or running
        self.contexts = []           # all live contexts
        self.free = []               # evicted contexts kept for reuse
        self.inflight = []           # (context, kind, [(request, k or None)])
        self.bytes_per_particle = 768.0   # predicted need, refined from gg_device_bytes
        self.fixed_bytes = 128 << 20      # walk stacks and other buffers independent of N
        self.threaded = threaded
        self._fetch_q, self._done_q = queue.Queue(), queue.Queue()
        self._worker = None
        self.fetching = 0            # launches finished on the device, results being copied out
        self.n_batches = 0
        self.evictions = 0
        self.peak_bytes = 0
        self.done = []

    # ---------------------------------------------------------------- memory
    def held_bytes(self):
        return sum(c.bytes for c in self.contexts)

    def _predict(self, n):
        return self.fixed_bytes + self.bytes_per_particle * n

    def _evict_one(self):
        idle = [c for c in self.contexts if not c.busy and c.sids]
        if not idle:
            return False
        victim = min(idle, key=lambda c: c.last_use)
        for sid in victim.sids:
            self.resident.pop(sid, None)
        victim.sids = []
        self.free.append(victim)
        self.evictions += 1
        return True

    def _drop_free(self):
        while self.free:
            c = self.free.pop()
            self.contexts.remove(c)
            c.tree.close()

    def _get_context(self, need):
        """A context for a batch needing `need` bytes, within the budget, or None."""
        while True:
            reuse = [c for c in self.free if c.bytes >= need]
            if reuse:
                c = min(reuse, key=lambda c: c.bytes)
                self.free.remove(c)
                return c
            grow = self.free[-1].bytes if self.free else 0
            if self.held_bytes() - grow + need <= self.budget:
                if self.free:
                    c = self.free.pop()
                    return c
                c = _Context(self.tree_factory(**self.cfg))
                self.contexts.append(c)
                return c
            if self.free:
                self._drop_free()
                continue
            if not self._evict_one():
                return None

    def _account(self, c, n):
        c.bytes = c.tree.device_bytes()
        if n > 0:
            self.bytes_per_particle = max(self.bytes_per_particle, (c.bytes - self.fixed_bytes) / n)
        self.peak_bytes = max(self.peak_bytes, self.held_bytes())

    # ---------------------------------------------------------------- requests
    def submit(self, req):
        if req.kind == "new":
            self.systems[req.rid] = req.system
            self.drifted[req.rid] = 0.0
            self.unsolved.add(req.rid)
            self.pending_new.append(req)
        else:
            self.pending_re.append(req)

    def _launch_new(self, reqs, now):
        n = sum(r.n for r in reqs)
        c = self._get_context(self._predict(n))
        if c is None:
            return False
        systems = []
        for r in reqs:
            s = r.system
            if r.kind == "reeval":            # a miss: the drifted system, solved afresh
                d = self.drifted[r.target]
                s = dict(s, pos=s["pos"] + s["vel"] * d)
            systems.append(s)
        t = c.tree
        t.load_systems(systems)
        t.build()
        t.evaluate_async(err_tol_theta=STARTUP_THETA, copy_acc=False, copy_pot=False)
        if self.pinned_results:
            t.evaluate_async_pinned(self.result_alloc((n, 3)), self.result_alloc(n), err_tol_force_acc=self.tol,
                                    err_tol_theta=0.0)
        else:
            t.evaluate_async(err_tol_force_acc=self.tol, err_tol_theta=0.0)
        c.sids = [r.rid if r.kind == "new" else r.target for r in reqs]
        c.offsets = np.concatenate([[0], np.cumsum([r.n for r in reqs])])
        c.busy = True
        c.last_use = now
        self._account(c, n)
        for k, r in enumerate(reqs):
            r.batch = self.n_batches
        self.inflight.append((c, "new", [(r, k) for k, r in enumerate(reqs)]))
        self.n_batches += 1
        return True

    def _launch_reeval(self, c, group, now):
        dts = np.zeros(len(c.sids))
        active = []
        items = []
        for r, k in group:
            dts[k] = r.dt
            lo, hi = c.range_of(k)
            active.append(np.arange(lo, hi, dtype=np.int32))
            items.append((r, k))
        t = c.tree
        t.drift(dts)
        act = np.concatenate(active)
        if self.pinned_results:
            t.evaluate_async_pinned(self.result_alloc((act.size, 3)), self.result_alloc(act.size), active=act,
                                    err_tol_force_acc=self.tol, err_tol_theta=0.0)
        else:
            t.evaluate_async(active=act, err_tol_force_acc=self.tol, err_tol_theta=0.0)
        c.busy = True
        c.last_use = now
        for r, k in group:
            self.drifted[r.target] += r.dt
            r.batch = self.n_batches
        self.inflight.append((c, "reeval", items))
        self.n_batches += 1

    def _fetch_loop(self):
        while True:
            job = self._fetch_q.get()
            if job is None:
                return
            c, kind, items = job
            try:
                res = c.tree.fetch()
                self._done_q.put((c, kind, items, res, time.perf_counter()))
            except Exception as e:   # handed to the scheduler thread
                self._done_q.put((c, kind, items, e, time.perf_counter()))

    def poll(self, now):
        """Collect finished work (`now`: the caller's clock, for the LRU order);
        returns the number of requests completed."""
        keep = []
        for c, kind, items in self.inflight:
            if not c.tree.query():
                keep.append((c, kind, items))
            elif self.threaded:
                if self._worker is None:
                    self._worker = threading.Thread(target=self._fetch_loop, daemon=True)
                    self._worker.start()
                self.fetching += 1
                self._fetch_q.put((c, kind, items))
            else:
                res = c.tree.fetch()
                self._done_q.put((c, kind, items, res, time.perf_counter()))
                self.fetching += 1
        self.inflight = keep
        done = 0
        while True:
            try:
                c, kind, items, res, t_fetched = self._done_q.get_nowait()
            except queue.Empty:
                break
            self.fetching -= 1
            done += self._finish(c, kind, items, res, t_fetched, now)
        return done

    def _finish(self, c, kind, items, res, t_fetched, now):
        if isinstance(res, Exception):
            raise res
        acc, pot, st = res
        if st["error_word"]:
            raise RuntimeError("device error word %d" % st["error_word"])
        done = 0
        off = 0
        for r, k in items:
            n = r.n
            r.acc, r.pot = acc[off:off + n], pot[off:off + n]   # views of this launch's fresh arrays
            off += n
            r.t_done = t_fetched
            self.done.append(r)
            done += 1
        if kind == "new":
            for k, sid in enumerate(c.sids):
                self.resident[sid] = (c, k)
                self.unsolved.discard(sid)
        c.busy = False
        c.last_use = now
        return done

    def schedule(self, now):
        """Admit waiting work while slots and memory allow."""
        # re-evaluations of resident, idle systems, grouped by context
        if self.pending_re:
            groups = collections.OrderedDict()
            waiting = collections.deque()
            for r in self.pending_re:
                sid = r.target
                if sid in self.resident:
                    c, k = self.resident[sid]
                    if c.busy or len(self.inflight) + len(groups) >= self.max_inflight and c not in groups:
                        waiting.append(r)
                        continue
                    g = groups.setdefault(c, [])
                    if any(k == kk for _, kk in g) or (not self.batching and g):
                        waiting.append(r)          # one drift of a system per launch
                        continue
                    r.n = c.range_of(k)[1] - c.range_of(k)[0]
                    g.append((r, k))
                elif self._target_pending(sid):
                    waiting.append(r)                # its system is not solved yet
                else:
                    r.miss = True                    # evicted: solve the drifted system afresh
                    r.system = self.systems[sid]
                    r.n = int(r.system["pos"].shape[0])
                    self.drifted[sid] += r.dt
                    self.unsolved.add(sid)
                    self.pending_new.appendleft(r)
            self.pending_re = waiting
            for c, g in groups.items():
                self._launch_reeval(c, g, now)
        # new systems, batched
        while self.pending_new and len(self.inflight) < self.max_inflight:
            reqs, n = [], 0
            for r in self.pending_new:
                if reqs and (n + r.n > self.max_batch_particles or len(reqs) >= self.max_batch_systems):
                    break
                reqs.append(r)
                n += r.n
            if not self._launch_new(reqs, now):
                if len(reqs) > 1:
                    reqs = reqs[:1]                  # a smaller batch may still fit
                    if self._launch_new(reqs, now):
                        self.pending_new.popleft()
                        continue
                if not self.inflight and self.held_bytes() == 0:
                    raise MemoryError("request %d needs more than the %.3g-byte budget" %
                                      (reqs[0].rid, self.budget))
                break
            for _ in reqs:
                self.pending_new.popleft()

    def _target_pending(self, sid):
        return sid in self.unsolved

    def idle(self):
        return not (self.pending_new or self.pending_re or self.inflight or self.fetching)

    def close(self):
        if self._worker is not None:
            self._fetch_q.put(None)
            self._worker.join()
            self._worker = None
        for c in self.contexts:
            c.tree.close()
        self.contexts = []
        self.free = []


def run_trace(server, requests, realtime=True, poll_sleep=50e-6):
    """Feed `requests` (sorted by arrival, seconds from the start) to `server`
    and drive it until every request is done.  Returns the wall time."""
    t0 = time.perf_counter()
    i, n = 0, len(requests)
    while i < n or not server.idle():
        now = time.perf_counter() - t0
        while i < n and (requests[i].arrival <= now or not realtime):
            r = requests[i]
            if not realtime:
                r.arrival = now
            server.submit(r)
            i += 1
        server.poll(now)
        server.schedule(now)
        if (server.inflight or server.fetching) and not server.pending_new and not server.pending_re:
            time.sleep(poll_sleep)
        elif not server.inflight and i < n:
            time.sleep(max(0.0, min(requests[i].arrival - (time.perf_counter() - t0), 1e-3)))
    for r in requests:
        r.t_done -= t0
    return time.perf_counter() - t0


def latency_stats(requests):
    lat = np.array([r.t_done - r.arrival for r in requests])
    parts = sum(r.n for r in requests)
    span = max(r.t_done for r in requests) - min(r.arrival for r in requests)
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "max_ms": float(lat.max() * 1e3), "requests": len(requests),
            "particles": int(parts), "makespan_s": float(span), "particles_per_s": parts / span}


def make_trace(pool, rate=2000.0, window_s=2.0, frac_reeval=0.3, dt=1e-3, recent=64, seed=20261205):
    """Poisson arrivals at `rate` per second over `window_s` seconds.  A new
    request takes a system of `pool` (a list of dicts with pos, vel, mass, h)
    chosen uniformly; with probability `frac_reeval` a request instead
    re-evaluates one of the `recent` latest new systems after a drift of dt."""
    rng = np.random.default_rng(seed)
    t, reqs, news = 0.0, [], []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window_s:
            break
        rid = len(reqs)
        if news and rng.uniform() < frac_reeval:
            target = news[-1 - int(rng.integers(0, min(recent, len(news))))]
            reqs.append(Request(rid, "reeval", t, target=target, dt=dt))
        else:
            reqs.append(Request(rid, "new", t, system=pool[int(rng.integers(0, len(pool)))]))
            news.append(rid)
    return reqs
