"""CPU checks of the drop-in boundary: the shared library loads, exports every
entry point include/fwix_b200.h declares, and rejects bad descriptors without a
GPU (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fwix_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(fwix_[a-z0-9_]+)\s*\(", src)))


def test_header_lists_entry_points():
    names = declared()
    assert "fwix_step" in names and "fwix_born" in names and len(names) >= 25


def test_library_exports_every_declared_symbol():
    from pyfwix_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from pyfwix_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared()


def test_invalid_descriptor_is_an_error_not_an_exit():
    from pyfwix_b200 import _lib
    lib = _lib.load()
    d = _lib.FwixDesc(nx=0, ny=4, nw=1, ns=1, nz=1, dx=1, dy=1, dz=1, nref=1)
    h = ctypes.c_void_p()
    st = lib.fwix_plan_create(ctypes.byref(d), ctypes.byref(h))
    assert st == -1 and not h.value
    assert b"positive" in lib.fwix_last_error()
    d = _lib.FwixDesc(nx=11 * 16, ny=4, nw=1, ns=1, nz=1, dx=1, dy=1, dz=1, nref=1)  # factor 11
    st = lib.fwix_plan_create(ctypes.byref(d), ctypes.byref(h))
    assert st == -2 and b"2^a 3^b 5^c" in lib.fwix_last_error()
    with pytest.raises(_lib.FwixError):
        _lib.check(-4)
