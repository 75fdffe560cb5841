"""The ctypes structs of the Python bindings have the C layout of include/b2c.h: a small C
program built against the header prints every struct's size and each field's offset, and they
equal the ctypes ones (a field added to one side only, or in another order, fails here)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

PAIRS = {"Bodies": "b2c_bodies", "Beads": "b2c_beads", "Grid": "b2c_grid", "Contacts": "b2c_contacts",
         "JacobiParams": "b2c_jacobi_params", "Manifold": "b2c_manifold", "Pairs": "b2c_pairs", "Warm": "b2c_warm",
         "Boxes": "b2c_boxes", "ColorParams": "b2c_color_params", "NcpScene": "b2c_ncp_scene",
         "NcpState": "b2c_ncp_state", "NcpParams": "b2c_ncp_params", "Bncp": "b2c_bncp", "Admm": "b2c_admm", "AdmmParams": "b2c_admm_params", "Config": "b2c_config",
         "StepHeader": "b2c_step_header", "World": "b2c_world"}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_header(me, tmp_path):
    L = me._lib
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "b2c.h"', "int main(void) {"]
    for py, c in PAIRS.items():
        cls = getattr(L, py)
        lines.append(f'printf("{py} size %zu\\n", sizeof({c}));')
        for name, *_ in cls._fields_:
            lines.append(f'printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines))
    r = subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(x.split()[:2]): int(x.split()[2]) for x in out if x.strip()}
    for py in PAIRS:
        cls = getattr(L, py)
        assert got[(py, "size")] == ctypes.sizeof(cls), py
        for name, *_ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)
