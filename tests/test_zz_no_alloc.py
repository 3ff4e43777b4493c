"""The allocation-free radix sort entry point (gg_radix_sort_pairs_noalloc).

It is for callers that cannot allocate device memory -- a process whose device
memory is already reserved in full by another allocator, or a latency-critical
loop that cannot take cudaFree's implicit synchronisation -- and uses the
library's static device scratch instead.  Checked through the C ABI against the
allocating entry point (gg_radix_sort_pairs) on two calls in a row: integer
work, so the results must be identical.  This file is collected last so that a
run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import ggb200

pytestmark = pytest.mark.gpu


def _fn():
    lib = ggb200.load_library()
    f = lib.gg_radix_sort_pairs_noalloc
    f.restype = ctypes.c_int32
    f.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
    return f


def _pairs(n, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 1 << 63, size=n, dtype=np.uint64)
    keys[: n // 4] = keys[n // 4: 2 * (n // 4)]   # duplicates
    keys[::5] &= np.uint64(0xFFFFF)
    return keys, np.arange(n, dtype=np.uint32)


def test_noalloc_sort_equals_allocating_sort_on_two_calls():
    import torch
    f = _fn()
    assert ggb200.NOALLOC_SORT_MAX_N == 1 << 20
    for call, (n, bits) in enumerate([(ggb200.NOALLOC_SORT_MAX_N, 64), (300007, 63)]):
        keys, vals = _pairs(n, 1000 + call)
        if bits < 64:
            keys &= np.uint64((1 << bits) - 1)
        k_ref = torch.from_numpy(keys.view(np.int64).copy()).cuda()
        v_ref = torch.from_numpy(vals.view(np.int32).copy()).cuda()
        ggb200.radix_sort_pairs(k_ref, v_ref, n, bits)
        k_new = torch.from_numpy(keys.view(np.int64).copy()).cuda()
        v_new = torch.from_numpy(vals.view(np.int32).copy()).cuda()
        st = f(n, k_new.data_ptr(), v_new.data_ptr(), bits, None)
        assert st == 0, ggb200.load_library().gg_strerror(st)
        torch.cuda.synchronize()
        assert torch.equal(k_new, k_ref) and torch.equal(v_new, v_ref), "call %d differs" % call
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(v_new.cpu().numpy().view(np.uint32), vals[order])


def test_noalloc_sort_rejects_sizes_beyond_its_limit():
    import torch
    f = _fn()
    k = torch.zeros(4, dtype=torch.int64, device="cuda")
    v = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert f(ggb200.NOALLOC_SORT_MAX_N + 1, k.data_ptr(), v.data_ptr(), 64, None) == -8   # GG_ERR_TOO_LARGE
    assert f(-1, k.data_ptr(), v.data_ptr(), 64, None) == -1


def test_noalloc_sort_rejects_host_pointers():
    """The pairs must be device memory of the current device, where the
    static array is; host memory is refused before any kernel runs."""
    f = _fn()
    keys, vals = _pairs(1000, 7)
    k0, v0 = keys.copy(), vals.copy()
    assert f(1000, keys.ctypes.data, vals.ctypes.data, 64, None) == -1   # GG_ERR_INVALID
    assert np.array_equal(keys, k0) and np.array_equal(vals, v0)
