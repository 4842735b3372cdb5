"""Drop-in for the reference's horizontal FCT correction (orbit/core/fct.py).

``compute_horizontal_fct_source(grid, indexer, c_flat, dt)`` (fct.py:459-492)
runs the two-pass Zalesak-limited anti-diffusive source on the device (K2)
and returns a host array like the reference.  ``fct_source_device`` keeps
everything on the device for the deferred-correction loop.
"""
from __future__ import annotations

import numpy as np

from .grid import met_from_griddata
from .synthetic import DTAU


def fct_source_device(met_device, c, dt=DTAU, limited=True):
    from . import device
    return device.fct_source(met_device, c, dt, limited)


def compute_horizontal_fct_source(grid, indexer, c_flat, dt, limited=True, c_ghost_flat=None):
    if c_ghost_flat is not None:
        raise NotImplementedError("lateral-inflow ghost cells are not supported by the device path")
    import torch
    from . import device
    md = device.MetDevice(met_from_griddata(grid))
    c = torch.as_tensor(np.asarray(c_flat, dtype=np.float64), device="cuda")
    return device.fct_source(md, c, dt, limited).cpu().numpy()
