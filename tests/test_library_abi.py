"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares."""
import glob
import os
import re

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"B2C_API\s+[^;(]*?\b(b2c_\w+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"b2c_version", "b2c_jacobi_substep", "b2c_body_predict"} <= names


def test_library_exports_every_declared_symbol(me):
    L = me._lib.load()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert L.b2c_version() >= 100


def test_bindings_cover_header(me):
    assert declared_symbols() <= set(me._lib.exported_symbols())


def test_bad_arguments_rejected_without_gpu(me):
    import ctypes
    L = me._lib.load()
    assert L.b2c_body_predict(None, ctypes.c_float(0.01), None) == 1
    assert b"bad" in L.b2c_last_error()
    assert L.b2c_exclusive_scan(None, None, 5, None, None) == 1


def test_grid_without_sorted_positions_rejected(me):
    """Every entry point that takes a bead grid checks all of its arrays, slot-ordered positions
    included, before touching the device."""
    import ctypes
    L = me._lib.load()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the check fails first
    g = me._lib.Grid(8, 8, 8, 0.1, dummy, dummy, dummy, dummy, dummy, None)
    beads = me._lib.Beads()
    assert L.b2c_grid_build(ctypes.byref(beads), ctypes.byref(g), None) == 1
    assert b"b2c_grid_build" in L.b2c_last_error()
    g.sorted_pos = dummy
    g.dim_z = 4  # below the 8 cells per axis the wrap-around query needs
    assert L.b2c_grid_build(ctypes.byref(beads), ctypes.byref(g), None) == 1
