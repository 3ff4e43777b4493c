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
    assert cfg.group_order == 1 and cfg.target_order == 1 and cfg.node_staging == 0 and ctypes.sizeof(cfg) == 40
    assert cfg.walk_stack_entries == 0
    cfg.leaf_size = 0
    h = ctypes.c_void_p()
    assert lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    lib.gg_config_default(ctypes.byref(cfg))
    cfg.group_order = 2
    assert lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    lib.gg_config_default(ctypes.byref(cfg))
    cfg.node_staging = 2
    assert lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    lib.gg_config_default(ctypes.byref(cfg))
    cfg.walk_stack_entries = -1
    assert lib.gg_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    assert lib.gg_radix_sort_pairs(-1, None, None, 64, None) == -1


def _header_struct(name):
    """(type, field, count) of `typedef struct name { ... } name;` in the public header."""
    import re
    here = os.path.dirname(ggb200.__file__)
    text = open(os.path.join(here, "..", "include", "gizmo_gravity_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(\w+)\s+(\w+)(?:\[(\d+)\])?$", decl)
        assert m, decl
        out.append((m.group(1), m.group(2), int(m.group(3) or 1)))
    return out


C_TYPES = {"int32_t": ctypes.c_int32, "int64_t": ctypes.c_int64, "double": ctypes.c_double}


def _mirror(fields):
    out = []
    for name, t in fields:
        if hasattr(t, "_length_"):   # array: element type and count
            out.append((t._type_, name, t._length_))
        else:
            out.append((t, name, 1))
    return out


def test_binding_structs_mirror_header():
    for cname, py in (("gg_config", ggb200.Config), ("gg_stats", ggb200.Stats), ("gg_domain", ggb200.Domain)):
        h = _header_struct(cname)
        m = _mirror(py._fields_)
        assert [f for _, f, _ in h] == [f for _, f, _ in m], cname
        for (ct, f, n), (pt, _, pn) in zip(h, m):
            assert ctypes.sizeof(C_TYPES[ct]) == ctypes.sizeof(pt) and n == pn, (cname, f)


def test_particle_record_layout():
    import numpy as np
    dt = ggb200.PART_DTYPE
    assert dt.itemsize == 32
    assert [(k, dt.fields[k][1]) for k in ("x", "y", "z", "m", "h")] == [("x", 0), ("y", 8), ("z", 16), ("m", 24),
                                                                         ("h", 28)]
    pos = np.arange(12, dtype=np.float64).reshape(4, 3) + 0.1
    rec = ggb200.make_records(pos, np.full(4, 0.25), np.full(4, 0.028))
    assert np.array_equal(np.stack([rec["x"], rec["y"], rec["z"]], 1), pos)
    assert rec["m"].dtype == np.float32 and np.all(rec["m"] == np.float32(0.25))
    assert np.all(rec["h"] == np.float32(0.028))
