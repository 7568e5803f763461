"""The C-ABI library builds, loads and exports exactly what include/*.h
declares.  No device calls (runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from pypaswas_b200 import _native

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(pw_[a-z_0-9]+)\s*\(", text))
    return names


def test_library_loads_and_exports_every_declared_symbol(engine_lib):
    lib = ctypes.CDLL(_native.LIBRARY_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_binding_covers_the_header():
    assert declared_functions() == set(_native.EXPORTED_SYMBOLS)


def test_struct_layouts_match_header():
    assert ctypes.sizeof(_native.PwHit) == 48
    assert _native.START_DTYPE.itemsize == 36  # StartingPoint, default_main.cu:66-76


def test_struct_field_offsets_match_the_c_compiler(tmp_path):
    """Every field of the ctypes mirrors sits at the offset the C compiler
    gives the header's struct (gcc on the header itself), and the sizes agree."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    pairs = [("pw_hit", _native.PwHit), ("pw_run_info", _native.PwRunInfo),
             ("pw_request_info", _native.PwRequestInfo), ("pw_server_counters", _native.PwServerStats)]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "paswas_b200.h"', "int main(void) {"]
    for cname, py in pairs:
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(REPO, "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line.strip():
            a, b, v = line.split()
            got[(a, b)] = int(v)
    for cname, py in pairs:
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
