"""The C ABI library loads and exports every entry point include/*.h declares
(no device calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(sfgpu_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "sfgpu_system_create" in names and "sfgpu_residual" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from field_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from field_b200 import _native
    missing = [n for n in declared_symbols() if n not in _native.PROTOTYPES]
    assert not missing, missing
