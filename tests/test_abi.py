"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import glob
import os
import re

from conftest import ROOT

from cudaraytracer_b200 import _lib


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(crt_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "crt_trace_closest" in names and "crt_trace_shadow" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"libcrt.so lacks {missing}"


def test_bindings_cover_header():
    assert set(declared_functions()) <= set(_lib._SIGS), "ctypes signatures missing for some entry points"


def test_version_string():
    assert _lib.lib().crt_version().decode().startswith("crt")
