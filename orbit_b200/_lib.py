"""ctypes binding of liborbit_b200.so (include/orbit_b200.h).

The shared library is built in-tree (``python -m orbit_b200.build``).  There
is no CPU fallback: importing this module without the library raises, and
every call that fails on the device raises ``RuntimeError`` with the
library's message, the way the reference raises on a non-zero UMFPACK status
(orbit/core/solve.py:197-198, 231-232, 275-276).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("ORBIT_B200_LIB") or os.path.join(HERE, "liborbit_b200.so")

ORBIT_OK = 0
ERR_NAMES = {1: "ORBIT_ERR_ARG", 2: "ORBIT_ERR_NOMEM", 3: "ORBIT_ERR_CUDA", 4: "ORBIT_ERR_TIMEOUT",
             5: "ORBIT_ERR_PIVOT", 6: "ORBIT_ERR_NOCONV", 7: "ORBIT_ERR_INTERNAL",
             8: "ORBIT_ERR_NOTFINITE"}
PREC_FP64 = 64
PREC_FP32 = 32


class OrbitError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class MetT(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "dP", "Dz", "u", "v", "u_plus", "u_minus", "v_plus", "v_minus", "u_e", "u_plus_e",
        "v_n", "v_plus_n", "kxxyy", "kzz", "w_plus", "w_minus", "cmfmc", "kmu", "kmv", "lat")] + [
        ("dlat", C.c_double), ("dlon", C.c_double), ("split", C.c_int), ("pressure_form", C.c_int),
        ("periodic_lon", C.c_int)] + [(n, C.c_void_p) for n in ("u_wrap", "u_plus_wrap", "u_minus_wrap", "kmu_wrap")]


class SpeciesFieldsT(C.Structure):
    """orbit_species_fields_t (include/orbit_b200.h)."""
    _fields_ = [(n, C.c_void_p) for n in (
        "Dz", "particle_dry_dep", "nh3_dry_dep", "so2_dry_dep", "nox_dry_dep", "hno3_dry_dep", "o3_dry_dep",
        "is_land", "voc_dry_dep", "particle_wet_dep", "other_gas_wet_dep", "so2_wet_dep", "nh_part",
        "no3_part", "fp_vbs", "fp_vbs_surface", "j_no2")] + [("a_photo", C.c_double)] + [
        (n, C.c_void_p) for n in ("so2_ox", "nox_ox", "o3_loss", "co_loss", "archive_oh")] + [
        ("k_age", C.c_double), ("aging_gain", C.c_double)]


class OxidantFieldsT(C.Structure):
    """orbit_oxidant_fields_t (include/orbit_b200.h)."""
    _fields_ = [(n, C.c_void_p) for n in ("temperature", "pressure", "oh", "no", "no2", "no3rad", "p_s", "p_nh",
                                          "p_no", "dust_fine", "sea_salt_fine")]


class LutT(C.Structure):
    """orbit_lut_t (include/orbit_b200.h)."""
    _fields_ = [("axis", C.c_void_p * 7), ("n", C.c_int * 7), ("field", C.c_void_p * 4)]


EXPORTS = {
    "orbit_last_error": (C.c_char_p, []),
    "orbit_version": (C.c_char_p, []),
    "orbit_kernel_launches": (C.c_longlong, []),
    "orbit_factor_profile": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "orbit_symbolic_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "orbit_symbolic_create_ex": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.c_void_p)]),
    "orbit_symbolic_create_grid": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.POINTER(C.c_void_p)]),
    "orbit_symbolic_destroy": (C.c_int, [C.c_void_p]),
    "orbit_symbolic_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.c_int]),
    "orbit_symbolic_perm": (C.c_int, [C.c_void_p, C.c_void_p]),
    "orbit_symbolic_array": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int64,
                                       C.POINTER(C.c_int64)]),
    "orbit_assemble_transport": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(MetT), C.c_void_p,
                                           C.c_void_p, C.c_void_p]),
    "orbit_transport_boundary_loss": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(MetT), C.c_void_p,
                                                C.c_void_p]),
    "orbit_mass_balance_rows": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]),
    "orbit_nox_to_no3_rate": (C.c_int, [C.c_int64, C.POINTER(OxidantFieldsT), C.c_int, C.c_void_p, C.c_void_p]),
    "orbit_species_diagonals": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(SpeciesFieldsT), C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    "orbit_source_coupling": (C.c_int, [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]),
    "orbit_lut_query": (C.c_int, [C.POINTER(LutT), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "orbit_vec_dots": (C.c_int, [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "orbit_vec_combine": (C.c_int, [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                    C.c_void_p]),
    "orbit_fct_source": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(MetT), C.c_int, C.c_void_p,
                                   C.c_double, C.c_int, C.c_void_p, C.c_void_p]),
    "orbit_fct_linear_operator": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_double,
                                            C.c_void_p, C.c_void_p]),
    "orbit_stencil_apply": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_double, C.c_int, C.c_void_p, C.c_void_p]),
    "orbit_fct_source_ghost": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(MetT), C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p]),
    "orbit_stencil_apply_grid": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                           C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p]),
    "orbit_fct_source_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(MetT), C.c_int,
                                           C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p]),
    "orbit_factor_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "orbit_factor_create_ex": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_void_p)]),
    "orbit_factor_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "orbit_factor_destroy": (C.c_int, [C.c_void_p]),
    "orbit_factor_numeric": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                       C.c_void_p]),
    "orbit_factor_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "orbit_chain_apply": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p]),
    "orbit_selftest_wait_timeout": (C.c_int, [C.c_void_p, C.c_void_p]),
    "orbit_gmres_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_void_p,
                                    C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p]),
    "orbit_adjoint_gmres_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                            C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
}

_lib = None


def lib():
    """Load the library once; raise loudly if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m orbit_b200.build` "
                              "(the device path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != ORBIT_OK:
        msg = lib().orbit_last_error().decode(errors="replace")
        raise OrbitError(rc, msg)


def ptr(t) -> int:
    """Raw device (or host) address of a torch tensor / numpy array, or 0 for None."""
    if t is None:
        return 0
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def ptr_array(ptrs):
    arr = (C.c_void_p * len(ptrs))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr
