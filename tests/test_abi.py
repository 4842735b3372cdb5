"""The C-ABI library loads and exports every symbol include/orbit_b200.h declares
(no device calls)."""
import ctypes
import os
import re

from orbit_b200 import _lib

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "orbit_b200.h")


def _declared():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(orbit_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_binding_covers_header():
    assert set(_declared()) <= set(_lib.EXPORTS)


def test_host_only_calls():
    L = _lib.lib()
    assert L.orbit_version().startswith(b"orbit_b200")
    h = ctypes.c_void_p()
    assert L.orbit_symbolic_create(0, 5, 5, 0, ctypes.byref(h)) == 1  # bad argument, no device touched
    assert b"positive" in L.orbit_last_error()
