"""ctypes handle on the CPU oracle (oracle/gg_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg load this module to check or time the CUDA library against a
plain-C FP64 restatement of GIZMO's tree-gravity algorithm.  The product path
never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force=False):
    if force or not os.path.exists(LIB):
        subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        P, i64, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        L.oracle_find_extent.argtypes = [i64, P, P, P, P]
        L.oracle_find_extent.restype = None
        L.oracle_double_to_int.argtypes = [dbl, ctypes.c_int]
        L.oracle_double_to_int.restype = ctypes.c_uint64
        L.oracle_ph_keys.argtypes = [i64, P, P, dbl, ctypes.c_int, P, P]
        L.oracle_ph_keys.restype = None
        L.oracle_spline_gravity.argtypes = [dbl, dbl, dbl, ctypes.c_int]
        L.oracle_spline_gravity.restype = dbl
        L.oracle_tree_gravity.argtypes = [i64, P, P, P, P, dbl, dbl, i64, P, P, P, P, ctypes.c_int]
        L.oracle_tree_gravity.restype = i64
        L.oracle_tree_gravity_drift.argtypes = [i64, P, P, P, P, P, dbl, dbl, dbl, i64, P, P, P, P, P, ctypes.c_int]
        L.oracle_tree_gravity_drift.restype = i64
        L.oracle_potential.argtypes = [i64, P, P, P, P, dbl, dbl, i64, P, P, ctypes.c_int]
        L.oracle_potential.restype = None
        L.oracle_tree_nodes.argtypes = [i64, P, P, P]
        L.oracle_tree_nodes.restype = i64
        L.oracle_direct_sum.argtypes = [i64, P, P, P, i64, P, P, P, ctypes.c_int]
        L.oracle_direct_sum.restype = None
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def find_extent(pos):
    pos = _c(pos, np.float64)
    c, k, ln = np.zeros(3), np.zeros(3), np.zeros(1)
    lib().oracle_find_extent(pos.shape[0], pos.ctypes.data, c.ctypes.data, k.ctypes.data, ln.ctypes.data)
    return dict(center=c.tolist(), corner=k.tolist(), len=float(ln[0]))


def ph_keys(pos, domain, bits=21):
    """Keys as Python ints (3*bits bits), via the restated key function."""
    pos = _c(pos, np.float64)
    n = pos.shape[0]
    hi, lo = np.zeros(n, np.uint64), np.zeros(n, np.uint64)
    corner = _c(domain["corner"], np.float64)
    lib().oracle_ph_keys(n, pos.ctypes.data, corner.ctypes.data, domain["len"], bits, hi.ctypes.data, lo.ctypes.data)
    return hi, lo


def spline_gravity(u, hinv, hinv3, mode):
    return lib().oracle_spline_gravity(u, hinv, hinv3, mode)


def tree_gravity(pos, mass, h, old_acc=None, err_tol_force_acc=0.0025, err_tol_theta=0.0, targets=None, nthreads=0):
    """GIZMO-semantics tree force (one pass).  Returns acc (pre-G), pot, ninter, total."""
    pos, mass, h = _c(pos, np.float64), _c(mass, np.float64), _c(h, np.float64)
    n = pos.shape[0]
    tg = None if targets is None else _c(targets, np.int32)
    nt = n if tg is None else tg.shape[0]
    oa = None if old_acc is None else _c(old_acc, np.float64)
    acc = np.zeros((nt, 3))
    pot = np.zeros(nt)
    nint = np.zeros(nt, np.int64)
    total = lib().oracle_tree_gravity(n, pos.ctypes.data, mass.ctypes.data, h.ctypes.data,
                                      None if oa is None else oa.ctypes.data, err_tol_force_acc, err_tol_theta, nt,
                                      None if tg is None else tg.ctypes.data, acc.ctypes.data, pot.ctypes.data,
                                      nint.ctypes.data, nthreads)
    return acc, pot, nint, int(total)


def tree_gravity_two_pass(pos, mass, h, err_tol_force_acc=0.0025, err_tol_theta=0.7, targets=None, nthreads=0):
    """GIZMO start-up evaluation (accel.c:47-50): BH pass for OldAcc, then relative pass."""
    a1, _, _, _ = tree_gravity(pos, mass, h, None, err_tol_force_acc, err_tol_theta, None, nthreads)
    old = np.linalg.norm(a1, axis=1)
    return tree_gravity(pos, mass, h, old, err_tol_force_acc, 0.0, targets, nthreads) + (old,)


def tree_gravity_drift(pos, vel, mass, h, dt, old_acc=None, err_tol_force_acc=0.0025, err_tol_theta=0.0,
                       targets=None, nthreads=0):
    """Tree built at `pos`, then particles and nodes drifted by dt without a
    rebuild (force_drift_node), then one pass at the drifted positions.
    Returns acc (pre-G), pot, ninter, total, drifted positions."""
    pos, vel = _c(pos, np.float64), _c(vel, np.float64)
    mass, h = _c(mass, np.float64), _c(h, np.float64)
    n = pos.shape[0]
    tg = None if targets is None else _c(targets, np.int32)
    nt = n if tg is None else tg.shape[0]
    oa = None if old_acc is None else _c(old_acc, np.float64)
    acc, pot, nint = np.zeros((nt, 3)), np.zeros(nt), np.zeros(nt, np.int64)
    moved = np.zeros((n, 3))
    total = lib().oracle_tree_gravity_drift(n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data, h.ctypes.data,
                                            None if oa is None else oa.ctypes.data, err_tol_force_acc, err_tol_theta,
                                            dt, nt, None if tg is None else tg.ctypes.data, acc.ctypes.data,
                                            pot.ctypes.data, nint.ctypes.data, moved.ctypes.data, nthreads)
    return acc, pot, nint, int(total), moved


def potential(pos, mass, h, old_acc=None, err_tol_force_acc=0.0025, err_tol_theta=0.0, targets=None, nthreads=0):
    """compute_potential: the potential-only walk with the self term removed (pre-G)."""
    pos, mass, h = _c(pos, np.float64), _c(mass, np.float64), _c(h, np.float64)
    n = pos.shape[0]
    tg = None if targets is None else _c(targets, np.int32)
    nt = n if tg is None else tg.shape[0]
    oa = None if old_acc is None else _c(old_acc, np.float64)
    pot = np.zeros(nt)
    lib().oracle_potential(n, pos.ctypes.data, mass.ctypes.data, h.ctypes.data, None if oa is None else oa.ctypes.data,
                           err_tol_force_acc, err_tol_theta, nt, None if tg is None else tg.ctypes.data, pot.ctypes.data,
                           nthreads)
    return pot


def tree_nodes(pos, mass, h):
    pos, mass, h = _c(pos, np.float64), _c(mass, np.float64), _c(h, np.float64)
    return int(lib().oracle_tree_nodes(pos.shape[0], pos.ctypes.data, mass.ctypes.data, h.ctypes.data))


def direct_sum(pos, mass, h, targets=None, nthreads=0):
    pos, mass, h = _c(pos, np.float64), _c(mass, np.float64), _c(h, np.float64)
    n = pos.shape[0]
    tg = None if targets is None else _c(targets, np.int32)
    nt = n if tg is None else tg.shape[0]
    acc = np.zeros((nt, 3))
    pot = np.zeros(nt)
    lib().oracle_direct_sum(n, pos.ctypes.data, mass.ctypes.data, h.ctypes.data, nt,
                            None if tg is None else tg.ctypes.data, acc.ctypes.data, pot.ctypes.data, nthreads)
    return acc, pot
