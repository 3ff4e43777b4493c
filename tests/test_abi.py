"""CPU checks of the C ABI library: it builds, loads and exports what the header declares."""
import ctypes
import os
import subprocess
import sys
import tempfile

import ggb200


def test_library_exports_every_declared_symbol():
    ggb200.build_library()
    lib = ctypes.CDLL(ggb200.LIB_PATH)
    names = ggb200.header_functions()
    assert "gg_evaluate" in names and "gg_build" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    lib = ggb200.load_library()
    for n in ggb200.header_functions():
        assert getattr(lib, n).argtypes is not None or getattr(lib, n).restype is None, n


def test_ph_table_header_is_generated():
    here = os.path.dirname(ggb200.__file__)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "t.h")
        subprocess.run([sys.executable, os.path.join(here, "gen_ph_tables.py"), out], check=True)
        assert open(out).read() == open(os.path.join(here, "csrc", "gg_ph_table.h")).read()


def test_strerror_and_no_device_error():
    lib = ggb200.load_library()
    assert lib.gg_strerror(-4) == b"node pool or walk stack overflow"
    import torch
    if not torch.cuda.is_available():
        cfg = ggb200.Config()
        lib.gg_config_default(ctypes.byref(cfg))
        h = ctypes.c_void_p()
        st = lib.gg_create(ctypes.byref(cfg), ctypes.byref(h))
        assert st == -2   # GG_ERR_CUDA: the library fails loudly without a device


def test_invalid_arguments_rejected_without_device():
    lib = ggb200.load_library()
    cfg = ggb200.Config()
    lib.gg_config_default(ctypes.byref(cfg))
    assert cfg.group_order == 1 and cfg.target_order == 1 and cfg.node_staging == 0 and ctypes.sizeof(cfg) == 36
    cfg.leaf_size = 0
    h = ctypes.c_void_p()
    assert lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    lib.gg_config_default(ctypes.byref(cfg))
    cfg.group_order = 2
    assert lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    lib.gg_config_default(ctypes.byref(cfg))
    cfg.node_staging = 2
    assert lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    assert lib.gg_radix_sort_pairs(-1, None, None, 64, None) == -1
