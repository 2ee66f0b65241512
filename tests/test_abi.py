"""The C-ABI library builds, loads and exports every symbol include/*.h
declares (no compute calls: this runs without a GPU)."""
import glob
import os
import re
import subprocess

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \t\*]*?\b((?:claw|nn)_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("claw_create", "claw_destroy", "claw_set_q", "claw_get_q", "claw_set_aux",
                 "claw_step", "claw_advance", "claw_advance_host"):
        assert must in names


def test_library_exports_every_declared_symbol(cuda_lib):
    from classic_b200 import _lib
    missing = [n for n in declared_symbols() if not hasattr(cuda_lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT ((?:claw|nn)_\w+)", out))
    assert declared_symbols() <= exported
    # the Python binding covers the whole ABI
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_library_is_built_for_sm100a(cuda_lib):
    from classic_b200 import build
    assert b"sm_100a" in cuda_lib.claw_build_info()
    assert "code=sm_100a" in build.ARCH


def test_config_struct_layout_matches_header(cuda_lib):
    """sizeof(claw_config) / sizeof(claw_stats) agree between C and ctypes."""
    import ctypes
    from classic_b200._lib import ClawConfig, ClawStats
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "s.c")
        open(c, "w").write('#include "claw_b200.h"\n#include <stdio.h>\n'
                           'int main(){printf("%zu %zu\\n", sizeof(claw_config), sizeof(claw_stats));}\n')
        exe = os.path.join(td, "s")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        a, b = map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split())
    assert a == ctypes.sizeof(ClawConfig)
    assert b == ctypes.sizeof(ClawStats)
