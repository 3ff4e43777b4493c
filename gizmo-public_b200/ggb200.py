"""Python binding (ctypes) of the B200 tree-gravity C ABI.

The entry points mirror GIZMO's gravity interface (gravity/gravtree.c
gravity_tree, gravity/forcetree.c force_treebuild / force_treeevaluate):
accelerations and potentials are returned in GIZMO's pre-G units and the
caller applies G (gravtree.c:495-501); OldAcc = |a|/G feeds the relative
opening criterion of the next pass (gravtree.c:514-522).

The CUDA library is required: every compute call raises GravityError when the
shared library or a CUDA device is missing.  There is no CPU fallback.
"""
import ctypes
import os
import re
import subprocess
import threading
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgizmo_gravity_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "gizmo_gravity_b200.h")

GG_OK = 0
GG_PENDING = 1
ASYNC_COPY_ACC, ASYNC_COPY_POT = 1, 2
ERRORS = {
    -1: "GG_ERR_INVALID", -2: "GG_ERR_CUDA", -3: "GG_ERR_NOMEM", -4: "GG_ERR_OVERFLOW",
    -5: "GG_ERR_TIMEOUT", -6: "GG_ERR_NOT_BUILT", -7: "GG_ERR_BAD_INPUT", -8: "GG_ERR_TOO_LARGE",
}

# one particle record on the device: {double x,y,z; float m; float h}
PART_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("m", "<f4"), ("h", "<f4")])
assert PART_DTYPE.itemsize == 32


class GravityError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = "%s (%d)" % (ERRORS.get(status, "unknown"), status)
        if _lib is not None:
            try:
                msg += ": " + _lib.gg_strerror(status).decode()
            except Exception:
                pass
        super().__init__((what + ": " if what else "") + msg)


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("leaf_size", ctypes.c_int32), ("group_size", ctypes.c_int32),
                ("flush_threshold", ctypes.c_int32), ("walk_blocks_per_sm", ctypes.c_int32),
                ("timing", ctypes.c_int32), ("target_order", ctypes.c_int32), ("group_order", ctypes.c_int32),
                ("node_staging", ctypes.c_int32), ("walk_stack_entries", ctypes.c_int32)]


class Domain(ctypes.Structure):
    _fields_ = [("center", ctypes.c_double * 3), ("corner", ctypes.c_double * 3), ("len", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("interactions", ctypes.c_int64), ("n_nodes", ctypes.c_int64), ("n_targets", ctypes.c_int64),
                ("n_groups", ctypes.c_int32), ("error_word", ctypes.c_int32), ("ms_keys", ctypes.c_double),
                ("ms_sort", ctypes.c_double), ("ms_build", ctypes.c_double), ("ms_walk", ctypes.c_double),
                ("far_entries", ctypes.c_int64), ("near_entries", ctypes.c_int64), ("nodes_tested", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_lock = threading.Lock()


def build_library(force=False):
    """Compile the CUDA library in-tree (nvcc, sm_100a)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-j8"], check=True, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return LIB_PATH


def header_functions():
    """Function names declared in include/gizmo_gravity_b200.h."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gg_[a-z0-9_]+)\s*\(", src)))


def load_library():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            build_library()
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        sig = {
            "gg_config_default": (None, [ctypes.POINTER(Config)]),
            "gg_create": (i32, [ctypes.POINTER(Config), ctypes.POINTER(P)]),
            "gg_destroy": (i32, [P]),
            "gg_strerror": (ctypes.c_char_p, [i32]),
            "gg_set_stream": (i32, [P, P]),
            "gg_synchronize": (i32, [P]),
            "gg_load_particles": (i32, [P, i32, P, P, i64, P, i64, P, i64]),
            "gg_load_particles_device": (i32, [P, i32, P, P]),
            "gg_build": (i32, [P, P]),
            "gg_get_domains": (i32, [P, P]),
            "gg_evaluate": (i32, [P, P, i64, P, dbl, dbl, P, P, P, ctypes.POINTER(Stats)]),
            "gg_evaluate_device": (i32, [P, P, i64, P, dbl, dbl, P, P, P]),
            "gg_last_stats": (i32, [P, ctypes.POINTER(Stats)]),
            "gg_peano_hilbert_keys": (i32, [i64, P, ctypes.POINTER(Domain), P, P]),
            "gg_radix_sort_pairs": (i32, [i64, P, P, i32, P]),
            "gg_direct_sum_fp64": (i32, [i64, P, P, P, i64, P, P, P, P]),
            "gg_fp32_peak_probe": (i32, [ctypes.POINTER(dbl), P]),
            "gg_radix_sort_pairs_noalloc": (i32, [i64, P, P, i32, P]),
            "gg_kernel_launches": (i64, []),
            "gg_selftest_bounded_wait": (i32, [P]),
            "gg_load_velocities": (i32, [P, P, i64]),
            "gg_load_velocities_device": (i32, [P, P]),
            "gg_drift": (i32, [P, dbl]),
            "gg_set_positions": (i32, [P, P, i64]),
            "gg_device_bytes": (i32, [P, ctypes.POINTER(i64)]),
            "gg_get_order": (i32, [P, P]),
            "gg_get_order_device": (i32, [P, P]),
            "gg_evaluate_potential": (i32, [P, P, i64, P, dbl, dbl, P, ctypes.POINTER(Stats)]),
            "gg_evaluate_potential_device": (i32, [P, P, i64, P, dbl, dbl, P]),
            "gg_energy_device": (i32, [P, P, P, P]),
            "gg_reserve_device_pool": (i32, [i32, i64]),
            "gg_load_systems": (i32, [P, i32, P, P, P, P]),
            "gg_load_system_velocities": (i32, [P, P]),
            "gg_evaluate_async": (i32, [P, P, i64, dbl, dbl, i32]),
            "gg_query": (i32, [P]),
            "gg_fetch_results": (i32, [P, P, P, ctypes.POINTER(Stats)]),
            "gg_evaluate_async_pinned": (i32, [P, P, i64, dbl, dbl, P, P]),
            "gg_host_alloc": (i32, [i64, ctypes.POINTER(P)]),
            "gg_host_free": (i32, [P]),
            "gg_drift_systems": (i32, [P, P]),
            "gg_graph_capture_step": (i32, [P, dbl, dbl, P, P]),
            "gg_graph_capture_parts": (i32, [P, dbl, dbl, P, P]),
            "gg_graph_launch_part": (i32, [P, i32]),
            "gg_graph_launch": (i32, [P]),
            "gg_autotune": (i32, [P, dbl, dbl, ctypes.POINTER(Config), ctypes.POINTER(dbl)]),
            "gg_tune_accuracy": (i32, [P, dbl, dbl, ctypes.POINTER(Config), ctypes.POINTER(i32)]),
            "gg_autotune_active": (i32, [P, P, i64, dbl, dbl, ctypes.POINTER(Config), ctypes.POINTER(dbl)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
        return lib


def _check(status, what=""):
    if status != GG_OK:
        raise GravityError(status, what)


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())   # torch tensor


def make_records(pos, mass, h):
    """Pack (N,3) positions, masses and kernel radii into device record layout."""
    pos = np.asarray(pos, dtype=np.float64)
    rec = np.empty(pos.shape[0], dtype=PART_DTYPE)
    rec["x"], rec["y"], rec["z"] = pos[:, 0], pos[:, 1], pos[:, 2]
    rec["m"] = np.asarray(mass, dtype=np.float64)
    rec["h"] = np.asarray(h, dtype=np.float64)
    return rec


def domain_to_dict(d):
    return dict(center=list(d.center), corner=list(d.corner), len=d.len)


class GravityTree:
    """One library context: particles of one or more systems, their trees, walks."""

    def __init__(self, leaf_size=8, group_size=32, flush=128, device=0, timing=False, blocks_per_sm=0, target_order=1,
                 group_order=1, node_staging=0, walk_stack_entries=0):
        lib = load_library()
        cfg = Config()
        lib.gg_config_default(ctypes.byref(cfg))
        cfg.device, cfg.leaf_size, cfg.group_size, cfg.flush_threshold = device, leaf_size, group_size, flush
        cfg.timing = 1 if timing else 0
        cfg.walk_blocks_per_sm = blocks_per_sm
        cfg.target_order = target_order
        cfg.group_order = group_order
        cfg.node_staging = node_staging
        cfg.walk_stack_entries = walk_stack_entries
        h = ctypes.c_void_p()
        _check(lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)), "gg_create")
        self._lib, self._h = lib, h
        self.n = 0
        self.counts = None
        self._pinned_out = None

    def close(self):
        if self._h:
            self._lib.gg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_ptr):
        _check(self._lib.gg_set_stream(self._h, stream_ptr), "gg_set_stream")

    def synchronize(self):
        _check(self._lib.gg_synchronize(self._h), "gg_synchronize")

    def load(self, pos, mass, h, counts=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        h = np.ascontiguousarray(h, dtype=np.float64)
        n = pos.shape[0]
        counts = np.asarray([n] if counts is None else counts, dtype=np.int64)
        _check(self._lib.gg_load_particles(self._h, len(counts), counts.ctypes.data, pos.ctypes.data, 24,
                                           mass.ctypes.data, 8, h.ctypes.data, 8), "gg_load_particles")
        self.n, self.counts = n, counts
        self._keep = (pos, mass, h, counts)

    def load_device(self, records, counts):
        """records: device buffer (torch uint8/any tensor) holding N 32-byte records."""
        counts = np.asarray(counts, dtype=np.int64)
        _check(self._lib.gg_load_particles_device(self._h, len(counts), counts.ctypes.data, _ptr(records)),
               "gg_load_particles_device")
        self.n, self.counts = int(counts.sum()), counts

    def build(self, domains=None):
        arr = None
        if domains is not None:
            arr = (Domain * len(domains))()
            for i, d in enumerate(domains):
                arr[i].center[:] = list(d["center"])
                arr[i].corner[:] = list(d["corner"])
                arr[i].len = d["len"]
        _check(self._lib.gg_build(self._h, arr), "gg_build")

    def domains(self):
        arr = (Domain * len(self.counts))()
        _check(self._lib.gg_get_domains(self._h, arr), "gg_get_domains")
        return [domain_to_dict(d) for d in arr]

    def evaluate(self, active=None, old_acc=None, err_tol_force_acc=0.0025, err_tol_theta=0.0, want_ninter=False,
                 out=None):
        """Walk the trees for `active` particles (None = all).  Returns (acc, pot, ninter|None, stats).
        out: optional (acc (n,3), pot (n)) float64 arrays to write into, reused across calls."""
        act = None
        if active is not None:
            act = np.ascontiguousarray(active, dtype=np.int32)
        nt = self.n if act is None else act.shape[0]
        if out is not None:
            acc, pot = out
            assert acc.shape == (nt, 3) and pot.shape == (nt,) and acc.dtype == np.float64 and pot.dtype == np.float64
            assert acc.flags.c_contiguous and pot.flags.c_contiguous
        else:
            acc = np.empty((nt, 3), dtype=np.float64)
            pot = np.empty(nt, dtype=np.float64)
        nint = np.empty(nt, dtype=np.int64) if want_ninter else None
        oa = None if old_acc is None else np.ascontiguousarray(old_acc, dtype=np.float64)
        st = Stats()
        _check(self._lib.gg_evaluate(self._h, None if act is None else act.ctypes.data, nt,
                                     None if oa is None else oa.ctypes.data, err_tol_force_acc, err_tol_theta,
                                     acc.ctypes.data, pot.ctypes.data, None if nint is None else nint.ctypes.data,
                                     ctypes.byref(st)), "gg_evaluate")
        return acc, pot, nint, st.as_dict()

    def evaluate_device(self, d_acc, d_pot=None, d_active=None, n_active=0, d_old_acc=None, err_tol_force_acc=0.0025,
                        err_tol_theta=0.0, d_ninter=None):
        _check(self._lib.gg_evaluate_device(self._h, _ptr(d_active), n_active, _ptr(d_old_acc), err_tol_force_acc,
                                            err_tol_theta, _ptr(d_acc), _ptr(d_pot), _ptr(d_ninter)),
               "gg_evaluate_device")

    def last_stats(self):
        st = Stats()
        _check(self._lib.gg_last_stats(self._h, ctypes.byref(st)), "gg_last_stats")
        return st.as_dict()

    def load_velocities(self, vel):
        """Per-particle velocities (N,3) in load order: host array or device tensor."""
        if isinstance(vel, np.ndarray):
            v = np.ascontiguousarray(vel, dtype=np.float64)
            _check(self._lib.gg_load_velocities(self._h, v.ctypes.data, 24), "gg_load_velocities")
        else:
            _check(self._lib.gg_load_velocities_device(self._h, _ptr(vel)), "gg_load_velocities_device")

    def load_systems(self, systems):
        """Load independent systems given as separate arrays: a sequence of
        dicts with pos (n,3), mass (n), h (n) and optionally vel (n,3)."""
        arrs = [(np.ascontiguousarray(x["pos"], dtype=np.float64), np.ascontiguousarray(x["mass"], dtype=np.float64),
                 np.ascontiguousarray(x["h"], dtype=np.float64)) for x in systems]
        S = len(arrs)
        counts = np.array([a[0].shape[0] for a in arrs], dtype=np.int64)
        ptrs = [(ctypes.c_void_p * S)(*[a[k].ctypes.data for a in arrs]) for k in range(3)]
        _check(self._lib.gg_load_systems(self._h, S, counts.ctypes.data, ptrs[0], ptrs[1], ptrs[2]), "gg_load_systems")
        self.n, self.counts = int(counts.sum()), counts
        self._keep = (arrs, ptrs, counts)
        if all("vel" in x for x in systems):
            vs = [np.ascontiguousarray(x["vel"], dtype=np.float64) for x in systems]
            vp = (ctypes.c_void_p * S)(*[v.ctypes.data for v in vs])
            _check(self._lib.gg_load_system_velocities(self._h, vp), "gg_load_system_velocities")
            self._keepv = (vs, vp)

    def evaluate_async(self, active=None, err_tol_force_acc=0.0025, err_tol_theta=0.0, copy_acc=True,
                       copy_pot=True):
        """Queue a walk (and the copy of its results to pinned host memory); returns at once."""
        act = None if active is None else np.ascontiguousarray(active, dtype=np.int32)
        flags = (ASYNC_COPY_ACC if copy_acc else 0) | (ASYNC_COPY_POT if copy_pot else 0)
        n = 0 if act is None else act.shape[0]
        _check(self._lib.gg_evaluate_async(self._h, None if act is None else act.ctypes.data, n, err_tol_force_acc,
                                           err_tol_theta, flags), "gg_evaluate_async")
        self._async_n = self.n if act is None else n
        self._async_flags = flags
        self._pinned_out = None

    def query(self):
        """True when the last asynchronous evaluation has finished."""
        st = self._lib.gg_query(self._h)
        if st == GG_PENDING:
            return False
        _check(st, "gg_query")
        return True

    def evaluate_async_pinned(self, acc, pot, active=None, err_tol_force_acc=0.0025, err_tol_theta=0.0):
        """Queue a walk whose results are copied straight into `acc` (n, 3) and
        `pot` (n), page-locked arrays from host_empty (either may be None);
        fetch() then only waits and returns them."""
        act = None if active is None else np.ascontiguousarray(active, dtype=np.int32)
        n = self.n if act is None else act.shape[0]
        for a, shape in ((acc, (n, 3)), (pot, (n,))):
            if a is not None and (a.dtype != np.float64 or a.shape != shape or not a.flags.c_contiguous):
                raise ValueError("pinned result array must be C-contiguous float64 of shape %s" % (shape,))
        _check(self._lib.gg_evaluate_async_pinned(self._h, None if act is None else act.ctypes.data, 0 if act is None
                                                  else n, err_tol_force_acc, err_tol_theta, _ptr(acc), _ptr(pot)),
               "gg_evaluate_async_pinned")
        self._async_n = n
        self._async_flags = 0
        self._pinned_out = (acc, pot)

    def fetch(self):
        """Wait for the last asynchronous evaluation; returns (acc, pot, stats)."""
        if self._pinned_out is not None:
            acc, pot = self._pinned_out
            self._pinned_out = None
            st = Stats()
            _check(self._lib.gg_fetch_results(self._h, None, None, ctypes.byref(st)), "gg_fetch_results")
            return acc, pot, st.as_dict()
        n = self._async_n
        acc = np.empty((n, 3)) if self._async_flags & ASYNC_COPY_ACC else None
        pot = np.empty(n) if self._async_flags & ASYNC_COPY_POT else None
        st = Stats()
        _check(self._lib.gg_fetch_results(self._h, _ptr(acc), _ptr(pot), ctypes.byref(st)), "gg_fetch_results")
        return acc, pot, st.as_dict()

    def evaluate_potential(self, active=None, old_acc=None, err_tol_force_acc=0.0025, err_tol_theta=0.0):
        """The potential-only walk (compute_potential), pre-G.  Returns (pot, stats)."""
        act = None if active is None else np.ascontiguousarray(active, dtype=np.int32)
        nt = self.n if act is None else act.shape[0]
        pot = np.empty(nt)
        oa = None if old_acc is None else np.ascontiguousarray(old_acc, dtype=np.float64)
        st = Stats()
        _check(self._lib.gg_evaluate_potential(self._h, None if act is None else act.ctypes.data, nt,
                                               None if oa is None else oa.ctypes.data, err_tol_force_acc,
                                               err_tol_theta, pot.ctypes.data, ctypes.byref(st)),
               "gg_evaluate_potential")
        return pot, st.as_dict()

    def evaluate_potential_device(self, d_pot, d_active=None, n_active=0, d_old_acc=None, err_tol_force_acc=0.0025,
                                  err_tol_theta=0.0):
        _check(self._lib.gg_evaluate_potential_device(self._h, _ptr(d_active), n_active, _ptr(d_old_acc),
                                                      err_tol_force_acc, err_tol_theta, _ptr(d_pot)),
               "gg_evaluate_potential_device")

    def energy_device(self, d_acc=None, d_pot=None):
        """Per system [W = 1/2 sum m phi, sum m ax, sum m ay, sum m az] in FP64 (pre-G)."""
        out = np.empty((len(self.counts), 4))
        _check(self._lib.gg_energy_device(self._h, _ptr(d_acc), _ptr(d_pot), out.ctypes.data), "gg_energy_device")
        return out

    def order(self):
        """Load index of every sorted position of the last build (Peano-Hilbert order)."""
        out = np.empty(self.n, dtype=np.int32)
        _check(self._lib.gg_get_order(self._h, out.ctypes.data), "gg_get_order")
        return out

    def order_device(self, d_order):
        """The same order into a device int32 tensor of N entries (asynchronous)."""
        _check(self._lib.gg_get_order_device(self._h, _ptr(d_order)), "gg_get_order_device")

    def device_bytes(self):
        """Device memory the context holds now."""
        v = ctypes.c_int64()
        _check(self._lib.gg_device_bytes(self._h, ctypes.byref(v)), "gg_device_bytes")
        return v.value

    def drift(self, dt):
        """Move particles and nodes of the resident tree by dt (a number), or by
        one dt per system (a sequence), without a rebuild."""
        if np.ndim(dt) == 0:
            _check(self._lib.gg_drift(self._h, float(dt)), "gg_drift")
        else:
            d = np.ascontiguousarray(dt, dtype=np.float64)
            _check(self._lib.gg_drift_systems(self._h, d.ctypes.data), "gg_drift_systems")

    def set_positions(self, pos):
        """The particles' current positions (N,3, load order) replace the
        resident ones; the tree and its nodes stay (call drift first for the
        nodes)."""
        p = np.ascontiguousarray(pos, dtype=np.float64)
        _check(self._lib.gg_set_positions(self._h, p.ctypes.data, 24), "gg_set_positions")

    def capture_step(self, d_acc, d_pot=None, err_tol_force_acc=0.0025, err_tol_theta=0.0):
        """Capture build + walk of every resident system as one CUDA graph (the
        context needs its own stream, see set_stream, and one uncaptured step)."""
        _check(self._lib.gg_graph_capture_step(self._h, err_tol_force_acc, err_tol_theta, _ptr(d_acc), _ptr(d_pot)),
               "gg_graph_capture_step")

    def launch_step(self):
        """Replay the captured step on the context's stream (asynchronous)."""
        _check(self._lib.gg_graph_launch(self._h), "gg_graph_launch")

    def capture_step_parts(self, d_acc, d_pot=None, err_tol_force_acc=0.0025, err_tol_theta=0.0):
        """Capture the same step as two CUDA graphs, the build and the walk."""
        _check(self._lib.gg_graph_capture_parts(self._h, err_tol_force_acc, err_tol_theta, _ptr(d_acc), _ptr(d_pot)),
               "gg_graph_capture_parts")

    def launch_step_part(self, part):
        """Replay part 0 (build) or 1 (walk) of the captured step (asynchronous)."""
        _check(self._lib.gg_graph_launch_part(self._h, part), "gg_graph_launch_part")

    def autotune(self, err_tol_force_acc=0.0025, err_tol_theta=0.0, d_active=None, n_active=0):
        """Pick leaf size, group size, blocks per SM, flush threshold and node
        staging by timing the walk of the resident systems (of the active
        targets d_active, a device int32 tensor, when given), refusing any
        candidate less accurate than the context's configuration; returns
        (config dict, ms)."""
        cfg = Config()
        ms = ctypes.c_double()
        if d_active is None:
            _check(self._lib.gg_autotune(self._h, err_tol_force_acc, err_tol_theta, ctypes.byref(cfg),
                                         ctypes.byref(ms)), "gg_autotune")
        else:
            _check(self._lib.gg_autotune_active(self._h, _ptr(d_active), int(n_active), err_tol_force_acc,
                                                err_tol_theta, ctypes.byref(cfg), ctypes.byref(ms)),
                   "gg_autotune_active")
        return dict(leaf_size=cfg.leaf_size, group_size=cfg.group_size, flush=cfg.flush_threshold,
                    blocks_per_sm=cfg.walk_blocks_per_sm, node_staging=cfg.node_staging), ms.value

    def tune_accuracy(self, err_tol_force_acc=0.0025, err_tol_theta=0.0, **candidate):
        """The autotuner's accuracy gate for one candidate configuration
        (leaf_size, group_size, flush, blocks_per_sm, node_staging, target_order,
        group_order; unset fields keep the context's defaults) against this
        context's own: True if the candidate passes."""
        cfg = Config()
        self._lib.gg_config_default(ctypes.byref(cfg))
        names = {"leaf_size": "leaf_size", "group_size": "group_size", "flush": "flush_threshold",
                 "blocks_per_sm": "walk_blocks_per_sm", "node_staging": "node_staging",
                 "target_order": "target_order", "group_order": "group_order"}
        for k, v in candidate.items():
            setattr(cfg, names[k], int(v))
        ok = ctypes.c_int32()
        _check(self._lib.gg_tune_accuracy(self._h, err_tol_force_acc, err_tol_theta, ctypes.byref(cfg),
                                          ctypes.byref(ok)), "gg_tune_accuracy")
        return bool(ok.value)


def gravity_tree(pos, mass, h, G=1.0, err_tol_force_acc=0.0025, err_tol_theta=0.7, active=None, tree=None,
                 **cfg):
    """GIZMO's start-up force evaluation (accel.c:47-50): a Barnes-Hut pass with
    ErrTolTheta (begrun.c:2368) gives OldAcc, then the relative pass with
    ErrTolForceAcc (begrun.c:2369).  Returns acc*G, pot*G, OldAcc, stats of the
    relative pass (gravtree.c:495-522)."""
    own = tree is None
    t = tree or GravityTree(**cfg)
    try:
        t.load(pos, mass, h)
        t.build()
        a1, _, _, _ = t.evaluate(active=None, err_tol_theta=err_tol_theta)
        old = np.linalg.norm(a1, axis=1)   # |a| in pre-G units == OldAcc (|a G| / G)
        acc, pot, nint, st = t.evaluate(active=active, old_acc=old, err_tol_force_acc=err_tol_force_acc,
                                        err_tol_theta=0.0)
        acc_active_old = np.linalg.norm(acc, axis=1)
        return acc * G, pot * G, acc_active_old, st
    finally:
        if own:
            t.close()


def peano_hilbert_keys(d_pos, n, domain, d_keys, stream=None):
    lib = load_library()
    d = Domain()
    d.center[:] = list(domain["center"])
    d.corner[:] = list(domain["corner"])
    d.len = domain["len"]
    _check(lib.gg_peano_hilbert_keys(n, _ptr(d_pos), ctypes.byref(d), _ptr(d_keys), stream), "gg_peano_hilbert_keys")


def radix_sort_pairs(d_keys, d_vals, n, key_bits=64, stream=None):
    lib = load_library()
    _check(lib.gg_radix_sort_pairs(n, _ptr(d_keys), _ptr(d_vals), key_bits, stream), "gg_radix_sort_pairs")


NOALLOC_SORT_MAX_N = 1 << 20


def radix_sort_pairs_noalloc(d_keys, d_vals, n, key_bits=64, stream=None):
    """Radix sort that uses the library's static device scratch (no allocation)."""
    lib = load_library()
    _check(lib.gg_radix_sort_pairs_noalloc(n, _ptr(d_keys), _ptr(d_vals), key_bits, stream),
           "gg_radix_sort_pairs_noalloc")


def direct_sum_fp64(d_pos, d_mass, d_h, n_src, d_targets, n_tgt, d_acc, d_pot, stream=None):
    lib = load_library()
    _check(lib.gg_direct_sum_fp64(n_src, _ptr(d_pos), _ptr(d_mass), _ptr(d_h), n_tgt, _ptr(d_targets), _ptr(d_acc),
                                  _ptr(d_pot), stream), "gg_direct_sum_fp64")


def host_empty(shape, dtype=np.float64):
    """A numpy array in a page-locked block of the library's host cache
    (gg_host_alloc); the block goes back to the cache when the array and every
    view of it are gone."""
    lib = load_library()
    dt = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dt.itemsize
    p = ctypes.c_void_p()
    _check(lib.gg_host_alloc(max(nbytes, 1), ctypes.byref(p)), "gg_host_alloc")
    buf = (ctypes.c_char * max(nbytes, 1)).from_address(p.value)
    weakref.finalize(buf, lib.gg_host_free, ctypes.c_void_p(p.value))
    return np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)


def reserve_device_pool(nbytes, device=0):
    """Grow the device's memory pool by nbytes once (see gg_reserve_device_pool)."""
    _check(load_library().gg_reserve_device_pool(int(device), int(nbytes)), "gg_reserve_device_pool")


def selftest_bounded_wait(stream=None):
    """Run the sort look-back's bounded-wait self-test; returns the status
    (GG_ERR_TIMEOUT, -5, is the expected result)."""
    return int(load_library().gg_selftest_bounded_wait(stream))


def fp32_peak_tflops(stream=None):
    lib = load_library()
    v = ctypes.c_double()
    _check(lib.gg_fp32_peak_probe(ctypes.byref(v), stream), "gg_fp32_peak_probe")
    return v.value


def kernel_launches():
    return int(load_library().gg_kernel_launches())
