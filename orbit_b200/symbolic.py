"""Symbolic analysis handle (host side).

``Symbolic(nz, ny, nx)`` is the counterpart of the reference's
``umfpack_symbolic(L)`` (orbit/core/solve.py:88-207): computed once per
domain shape and reused for every species, bin and met draw.  Where the
reference derives an ordering from a sample matrix's pattern (COLAMD, or
METIS through pymetis), this analysis is geometric nested dissection of the
(nz, ny, nx) box into dense supernodes; the pattern is the full 7-point
stencil, so no sample matrix is needed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

_INT64_ARRAYS = {"ginv_off", "uoff", "fac_off", "front_off", "level_front_size", "ent_level_off", "ent_pos", "woff"}

INFO_KEYS = ("N", "nsuper", "nlevels", "factor_nnz", "factor_elems", "front_elems", "max_front",
             "factor_flops", "solve_items_per_bin", "update_len", "leaf_cells", "max_nm",
             "max_sub_front", "tc_pack_floats", "fused_fronts")


class Symbolic:
    def __init__(self, nz: int, ny: int, nx: int, leaf_cells: int = 0, chunk_elems: int = 0,
                 tc_min_n: int = 0, subtree_div: int = -1, periodic: bool = False):
        """Options left at 0 (subtree_div at -1) take the ORBIT_B200_* environment
        setting or the library default; `Symbolic.tuned` fills them from the
        autotuner's cache.  ``periodic``: the grid wraps in longitude
        (GridData.periodic_lon)."""
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check(L.orbit_symbolic_create_grid(int(nz), int(ny), int(nx), int(bool(periodic)), int(leaf_cells),
                                                int(chunk_elems), int(tc_min_n), int(subtree_div), C.byref(h)))
        self.periodic = bool(periodic)
        self.options = {"leaf_cells": int(leaf_cells), "chunk_elems": int(chunk_elems),
                        "tc_min_n": int(tc_min_n), "subtree_div": int(subtree_div)}
        self._h = h
        self.nz, self.ny, self.nx = int(nz), int(ny), int(nx)
        self.N = self.nz * self.ny * self.nx
        buf = (C.c_int64 * len(INFO_KEYS))()
        _lib.check(L.orbit_symbolic_info(h, buf, len(INFO_KEYS)))
        self.info = {k: int(buf[i]) for i, k in enumerate(INFO_KEYS)}

    @property
    def handle(self):
        return self._h

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    @property
    def lunz(self) -> int:
        """Structural nonzeros of one factor (sum over supernodes of n^2 + 2 n m)."""
        return self.info["factor_nnz"]

    def array(self, name: str) -> np.ndarray:
        L = _lib.lib()
        cnt = C.c_int64()
        _lib.check(L.orbit_symbolic_array(self._h, name.encode(), None, 0, C.byref(cnt)))
        dt = np.int64 if name in _INT64_ARRAYS else np.int32
        out = np.empty(cnt.value, dtype=dt)
        _lib.check(L.orbit_symbolic_array(self._h, name.encode(), out.ctypes.data, cnt.value,
                                          C.byref(cnt)))
        return out

    @classmethod
    def tuned(cls, nz: int, ny: int, nx: int, precision: int = 32, batch: int = 12,
              periodic: bool = False) -> "Symbolic":
        """Analysis with the autotuner's cached options for this device, shape,
        precision and (nearest) batch width; the defaults if none are cached."""
        from .autotune import tuned_options
        return cls(nz, ny, nx, periodic=periodic, **tuned_options((nz, ny, nx), precision, batch))

    def perm(self) -> np.ndarray:
        return self.array("perm")

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().orbit_symbolic_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
