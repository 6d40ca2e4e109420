"""The C-ABI library loads and exports every entry point include/n3ds.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from neural3dstrokes_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "n3ds.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(n3ds_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding covers every declared function
    assert set(names) <= set(_lib.EXPORTED), set(names) - set(_lib.EXPORTED)


def test_pure_host_calls():
    lib = _lib.load()
    assert lib.n3ds_version() >= 100
    assert lib.n3ds_stroke_workspace_bytes(1000) >= 1000 * 256
    assert lib.n3ds_compose_workspace_bytes(10, 20, 0) == 10 * 1 * 4  # one float per row and 32 strokes
    assert lib.n3ds_compose_workspace_bytes(10, 70, 0) == 10 * 3 * 4
    assert lib.n3ds_compose_workspace_bytes(10, 20, 1) == 0
    o = _lib.default_options()
    assert abs(o.cull_alpha - 1e-9) < 1e-15 and o.grad_mode == 0
    nr = (ctypes.c_int64 * 2)(100, 0)
    ns = (ctypes.c_int32 * 2)(5, 7)
    b = _lib.Batch(2, nr, ns, 64)
    assert lib.n3ds_field_workspace_bytes(ctypes.byref(b), ctypes.byref(o)) > 100 * 64 * 4 * 18
    bad = _lib.Batch(0, nr, ns, 64)
    assert lib.n3ds_field_workspace_bytes(ctypes.byref(bad), ctypes.byref(o)) == 0
    # argument validation happens before any device work
    rc = lib.n3ds_stroke_forward(None, None, None, None, 20, None, None, None, None, None, 10, 1, 4, 9, 3, 0x37, 0,
                                 0.02, 1, 1, None, 0, None)
    assert rc == 1 and b"texcoord" in lib.n3ds_last_error()
    rc = lib.n3ds_stroke_forward(None, None, None, None, 0, None, None, None, None, None, 10, 1, 4, 9, 3, 0x37, 3,
                                 0.02, 1, 1, None, 0, None)
    assert rc == 1 and b"27 columns" in lib.n3ds_last_error()
    rc = lib.n3ds_stroke_forward(None, None, None, None, 0, None, None, None, None, None, 10, 1, 4, 4, 3, 0xC0, 0,
                                 0.02, 1, 1, None, 0, None)
    assert rc in (1, 2)  # sdf base 12 does not exist
