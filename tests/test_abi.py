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


def test_argument_checks_of_the_grid_entry_points():
    """Host-side argument checks of the periodic-grid, boundary-loss, FCT
    inflow-field and NOx-rate entry points (ORBIT_ERR_ARG before any device
    work; the periodic analysis itself runs on the host)."""
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.orbit_symbolic_create_grid(3, 4, 2, 1, 4, 0, 0, -1, ctypes.byref(h)) == 1
    assert b"3 columns" in L.orbit_last_error()
    assert L.orbit_symbolic_create_grid(3, 4, 5, 1, 4, 0, 0, -1, ctypes.byref(h)) == 0
    assert L.orbit_symbolic_destroy(h) == 0
    met = _lib.MetT()
    assert L.orbit_transport_boundary_loss(3, 4, 5, None, None, None) == 1
    assert L.orbit_transport_boundary_loss(3, 4, 5, ctypes.byref(met), None, None) == 1
    assert L.orbit_fct_source_ghost(3, 4, 5, ctypes.byref(met), 1, None, None, 10800.0, 1, None, None) == 1
    assert L.orbit_stencil_apply_grid(3, 4, 2, 1, 1, None, None, 1.0, 0.0, 0, None, None) == 1
    ox = _lib.OxidantFieldsT()
    assert L.orbit_nox_to_no3_rate(60, ctypes.byref(ox), 0, None, None) == 1
    assert b"required field" in L.orbit_last_error()
    met.periodic_lon = 1
    T = ctypes.c_void_p(16)  # never dereferenced: the check fails first
    assert L.orbit_assemble_transport(3, 4, 5, ctypes.byref(met), T, None, None) == 1
