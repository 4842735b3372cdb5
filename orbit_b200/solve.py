"""Drop-in for the reference's factorization backend (orbit/core/solve.py).

The reference factors each ``I + dtau L`` with UMFPACK through ctypes, behind
a symbolic analysis computed once per run (``umfpack_symbolic``,
solve.py:88-207) and a numeric object with ``.solve(b, trans)``
(``_UmfpackLU``, solve.py:210-288).  Here the symbolic is the geometric
nested dissection of the grid (``orbit_b200.symbolic.Symbolic``) and the
numeric object is ``DeviceLU``: its factorization and triangular solves run
in liborbit_b200 on the GPU; ``.solve`` takes and returns host float64
arrays exactly like ``_UmfpackLU.solve``.

The module keeps the reference's flags so drivers that branch on them take
the factor-reuse path: ``_HAS_UMFPACK`` is True (the device LU plays
UMFPACK's role), ``_HAS_METIS`` False (the nested dissection is built in).
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from .grid import infer_grid_shape, infer_periodic, stencil_from_matrix
from .symbolic import Symbolic
from .synthetic import DTAU

_HAS_UMFPACK = True
_HAS_METIS = False
_UMFPACK_A = 0
_UMFPACK_At = 1

_default_shape = None


def set_grid_shape(nz: int, ny: int, nx: int) -> None:
    """Grid shape to use when an operator's pattern does not determine it."""
    global _default_shape
    _default_shape = (int(nz), int(ny), int(nx))


class DeviceSymbolic(dict):
    """The dict-like handle ``umfpack_symbolic`` returns (keys as in the reference:
    'n', 'lunz_est', 'strategy_used', 'ordering_used'), carrying the Symbolic."""

    @property
    def sym(self) -> Symbolic:
        return self["sym"]


def umfpack_symbolic(L, verbose: bool = True, ordering=None, qinit=None, grid_shape=None):
    """Symbolic analysis for every operator sharing L's 7-point pattern.

    ``ordering`` and ``qinit`` are accepted for signature compatibility and
    ignored: the ordering is the geometric nested dissection of the grid.
    The grid shape comes from ``grid_shape``, else from the pattern of L
    (off-diagonal offsets 1, nx, nx*ny), else from ``set_grid_shape``; a
    periodic-longitude grid is recognised by L's wrap-face couplings between
    columns 0 and nx-1.
    """
    shape = grid_shape or infer_grid_shape(L) or _default_shape
    if shape is None:
        raise ValueError("cannot determine the grid shape from L; pass grid_shape= or call set_grid_shape")
    sym = Symbolic(*shape, periodic=infer_periodic(L, tuple(shape)))
    if sym.N != L.shape[0]:
        raise ValueError(f"grid {shape} has {sym.N} cells, L has {L.shape[0]} rows")
    if verbose:
        print(f"  device symbolic (nested dissection {shape}): {sym.info['nsuper']} supernodes, "
              f"nnz(LU) {sym.lunz:,}")
    return DeviceSymbolic(sym=sym, n=sym.N, lunz_est=float(sym.lunz), strategy_used=3, ordering_used=-1,
                          shape=shape)


def umfpack_free_symbolic(symbolic) -> None:
    if symbolic and "sym" in symbolic:
        symbolic["sym"].close()


def compute_metis_ordering(L, verbose: bool = True):
    """Not needed: the device symbolic carries its own nested dissection."""
    raise ImportError("METIS is not used by the device path; umfpack_symbolic builds the ordering")


class DeviceLU:
    """``A = I + dtau L`` factored on the GPU; ``.solve(b, trans)`` as ``_UmfpackLU``.

    The factorization is done on first use (``solve``), or together with the
    other bins when eight of these are handed to ``solve_orbit_one_species``,
    which factors them in one batched launch sequence; from then on ``solve``
    uses the batch's factors (a lone factorization made earlier is released),
    so each LU's factors are held once.  Every ``solve`` moves b and x between
    host and device, as the reference's duck type takes and returns host
    arrays.
    """

    def __init__(self, L, symbolic, dtau: float = DTAU, precision: int = 64):
        sym = symbolic.sym if isinstance(symbolic, DeviceSymbolic) else symbolic
        if not isinstance(sym, Symbolic):
            raise TypeError("DeviceLU needs the handle returned by umfpack_symbolic")
        self.sym = sym
        self.dtau = float(dtau)
        self.precision = int(precision)
        self.stencil = stencil_from_matrix(L, sym.nz, sym.ny, sym.nx, periodic=getattr(sym, "periodic", False))
        self.shape = (sym.N, sym.N)
        self.numeric_bytes = float(sym.info["factor_elems"] * (8 if precision == 64 else 4))
        self.peak_bytes = float(sym.info["front_elems"] * 2 * (8 if precision == 64 else 4))
        self._fb = None
        self._T = None
        # after a bin-set factorization (solve_orbit_one_species): the batch
        # holding this LU's factors and its bin there
        self._set_fb = None
        self._set_bin = 0

    @property
    def nnz(self) -> int:
        return self.sym.lunz

    def device_stencil(self):
        import torch
        if self._T is None:
            self._T = torch.as_tensor(self.stencil, device="cuda")
        return self._T

    def attach_to_set(self, fb, bin_index: int):
        """Solve through bin ``bin_index`` of the batch ``fb`` from now on and
        release this LU's own factorization, if it had one: one set of factors
        per LU, whichever call factored it first."""
        self._set_fb = fb
        self._set_bin = int(bin_index)
        if self._fb is not None:
            self._fb.close()
            self._fb = None

    def _factored(self):
        if self._set_fb is not None:
            return self._set_fb
        if self._fb is None:
            from .device import FactorBatch
            fb = FactorBatch(self.sym, 1, self.precision, n_sets=1, n_bins=1)
            fb.numeric([self.device_stencil()], None, self.dtau)
            self._fb = fb
        return self._fb

    def solve(self, b: np.ndarray, trans: str = "N") -> np.ndarray:
        if trans not in ("N", "T"):
            raise ValueError(f"trans must be 'N' or 'T'; got {trans!r}")
        import torch
        fb = self._factored()
        t0 = self._set_bin if self._set_fb is not None else 0
        x = torch.as_tensor(np.ascontiguousarray(b, dtype=np.float64), device="cuda")[None]
        y = fb.chain(x, trans=(trans == "T"), tau0=t0, tau1=t0 + 1, refine=False)
        return y[0].cpu().numpy()


class _UmfpackLU(DeviceLU):
    """Name-compatible alias of DeviceLU (reference solve.py:210)."""

    def __init__(self, A, symbolic):
        # the reference's _UmfpackLU receives A = I + dtau L itself; with dtau = 1
        # the device assembles 1 + (A_ii - 1) on the diagonal and A_ij elsewhere
        super().__init__(A, symbolic, dtau=1.0)
        self.stencil[0] -= 1.0


def _splu(L, perm=None):
    raise RuntimeError("the device path has no SuperLU fallback; build a symbolic with umfpack_symbolic")
