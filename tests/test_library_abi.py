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
