"""Drop-in for the reference's horizontal FCT correction (orbit/core/fct.py).

``compute_horizontal_fct_source(grid, indexer, c_flat, dt[, c_ghost_flat])`` (fct.py:459-492)
runs the two-pass Zalesak-limited anti-diffusive source on the device (K2)
and returns a host array like the reference.  ``fct_source_device`` keeps
everything on the device for the deferred-correction loop.
``assemble_fct_linear_operator(grid, indexer, c_baseline_flat, dt)``
(fct.py:495-572) builds the frozen-gain operator L_AD on the device and
returns it as the reference's CSC matrix; ``fct_linear_operator_device``
keeps it as a 7-point stencil that adds to a transport stencil.
"""
from __future__ import annotations

import numpy as np

from .grid import met_from_griddata
from .synthetic import DTAU


def fct_source_device(met_device, c, dt=DTAU, limited=True):
    from . import device
    return device.fct_source(met_device, c, dt, limited)


def compute_horizontal_fct_source(grid, indexer, c_flat, dt, limited=True, c_ghost_flat=None):
    """``c_ghost_flat``: the lateral boundary inflow concentration, whose
    edge-cell values stand for the cells beyond each lateral edge (fct.py:283-292)."""
    import torch
    from . import device
    md = device.MetDevice(met_from_griddata(grid))
    c = torch.as_tensor(np.asarray(c_flat, dtype=np.float64), device="cuda")
    gh = None if c_ghost_flat is None else torch.as_tensor(np.asarray(c_ghost_flat, dtype=np.float64), device="cuda")
    return device.fct_source(md, c, dt, limited, c_ghost=gh).cpu().numpy()


def fct_linear_operator_device(met_device, c_base, dt=DTAU):
    from . import device
    return device.fct_linear_operator(met_device, c_base, dt)


def assemble_fct_linear_operator(grid, indexer, c_baseline_flat, dt):
    import torch
    from . import device
    md = device.MetDevice(met_from_griddata(grid))
    c = torch.as_tensor(np.asarray(c_baseline_flat, dtype=np.float64), device="cuda")
    st = device.fct_linear_operator(md, c, dt).cpu().numpy()
    nz, ny, nx = md.nz, md.ny, md.nx
    return device.stencil_to_csr(st, nz, ny, nx).tocsc()
