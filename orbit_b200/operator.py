"""Drop-in for the reference's transport assembly and air-mass-balance gate
(orbit/core/operator.py).

``assemble_transport_block(grid, indexer)`` (operator.py:281-347) assembles
the concentration-form block on the device (K1) and returns it as the
reference does, a scipy CSC matrix; ``transport_stencil(grid)`` returns the
device-resident [7, N] stencil the factorization consumes directly.
``mass_balance_diagnostics(grids, indexer)`` (operator.py:598-652) computes
the row sums on the device (K7) and the same order statistics; ``gate``
applies the reference's abort rule (cli.py:1590-1615: p90 > tol aborts).
Species diagonals (deposition and first-order chemistry, operator.py:371-595)
are per-cell bookkeeping and are taken as arrays (``species_operator``).
"""
from __future__ import annotations

import numpy as np

from .grid import met_from_griddata

MASS_BALANCE_TOL = 0.05  # per day (cli.py:161)


def transport_stencil(grid, with_rowsum=False):
    from . import device
    md = device.MetDevice(met_from_griddata(grid))
    return device.assemble_transport(md, with_rowsum=with_rowsum)


def assemble_transport_block(grid, indexer=None, scheme: str = "exp", return_boundary_fluxes: bool = False):
    if scheme != "exp":
        raise ValueError(f"Only the Patankar exponential scheme is supported (got scheme={scheme!r})")
    if return_boundary_fluxes:
        raise NotImplementedError("return_boundary_fluxes is not provided by the device path")
    from .device import stencil_to_csr
    T = transport_stencil(grid).cpu().numpy()
    return stencil_to_csr(T, int(grid.nz), int(grid.ny), int(grid.nx)).tocsc()


def species_operator(T, sink_diag):
    """L_s = T + diag(d_s) (operator.py:572-585) for a host CSC T."""
    import scipy.sparse as sp
    N = T.shape[0]
    return (T + sp.diags(np.asarray(sink_diag, dtype=np.float64), 0, shape=(N, N))).tocsc()


def mass_balance_diagnostics(grids, indexer=None, blocks=("transport",)) -> dict:
    from . import device
    mets = [device.MetDevice(met_from_griddata(g)) for g in grids]
    Ts = [device.assemble_transport(m) for m in mets]
    out = device.mass_balance(mets, Ts)
    out["units"] = "per day, |row sum| of the transport block, laterally interior cells, all bins"
    return out


def gate(diag: dict, tol: float = MASS_BALANCE_TOL) -> bool:
    """True when the air-mass balance passes (interior p90 <= tol per day)."""
    return not (diag["interior_p90"] > tol)
