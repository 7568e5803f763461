"""The C-ABI library builds, loads and exports exactly what include/*.h
declares.  No device calls (runs without a GPU)."""
import ctypes
import glob
import os
import re

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
