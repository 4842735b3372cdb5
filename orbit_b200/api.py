"""Batched periodic-orbit solver: the library's public entry point for many
orbits of one domain shape.

``OrbitSolver(nz, ny, nx, n_orbits, precision)`` keeps the symbolic
analysis, the factor storage and all work buffers resident on the device and
solves up to ``n_orbits`` orbits per call: the eight transport blocks are
assembled from the bin meteorology (K1), the n_orbits x 8 operators
``I + dtau (T + diag(sink))`` are factored (K3), and the periodic orbits are
found by batched GMRES over the chained solves (K4/K5).  It is the batched
form of the reference's per-species loop in ``solve_orbit_all_species``
(orbit/core/orbit.py:468-806) for species without cross-couplings.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np
import torch

from . import device
from .symbolic import Symbolic
from .synthetic import DTAU, N_BINS, MetBin, SpeciesFields


class OrbitSolver:
    def __init__(self, nz: int, ny: int, nx: int, n_orbits: int, precision: int = 64,
                 leaf_cells: int = 0, sym: Optional[Symbolic] = None):
        self.sym = sym if sym is not None else Symbolic(nz, ny, nx, leaf_cells)
        self.N = self.sym.N
        self.n_orbits = int(n_orbits)
        self.precision = int(precision)
        self.fb = device.FactorBatch(self.sym, self.n_orbits, self.precision)
        self._met_dev: List[device.MetDevice] = []
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    # -- device-resident path ------------------------------------------------
    def factor(self, T_stencils: Sequence[torch.Tensor], sinks: Sequence[torch.Tensor],
               n: int, dtau: float = DTAU):
        """T_stencils: 8 bin stencils shared by all orbits, or n*8 (orbit-major)."""
        if len(T_stencils) == N_BINS:
            T_list = [T_stencils[b] for _ in range(n) for b in range(N_BINS)]
        else:
            T_list = list(T_stencils)
        self.fb.numeric(T_list, list(sinks), dtau)

    def solve_device(self, E: torch.Tensor, tol: float, maxiter: int = 200, restart: int = 30,
                     c_warm: Optional[torch.Tensor] = None):
        return self.fb.solve(E, c_warm=c_warm, tol=tol, maxiter=maxiter, restart=restart)

    # -- host-facing path ----------------------------------------------------
    def solve(self, met: Sequence[MetBin], species: Sequence[SpeciesFields], tol: float = 1e-6,
              maxiter: int = 200, restart: int = 30, out: Optional[np.ndarray] = None):
        """Host arrays in, host orbits out: (n, 9, N) float64 and a list of info dicts."""
        n = len(species)
        if n > self.n_orbits:
            raise ValueError(f"at most {self.n_orbits} orbits per call")
        mets = [device.MetDevice(g) for g in met]
        self.h2d_bytes += sum(int(t.numel()) * 8 for m in mets for t in m.t.values())
        T = [device.assemble_transport(m) for m in mets]
        sinks = []
        for s in species:
            d = torch.as_tensor(s.sink_diag(met), device="cuda")
            sinks += [d[b] for b in range(N_BINS)]
        E = torch.as_tensor(np.stack([s.emis for s in species]), device="cuda")
        self.h2d_bytes += (n * N_BINS * self.N * 8) * 2
        self.factor(T, sinks, n)
        orb, info = self.fb.solve(E, tol=tol, maxiter=maxiter, restart=restart)
        if out is None:
            out = np.empty((n, N_BINS + 1, self.N))
        out[:n] = orb.cpu().numpy()
        self.d2h_bytes += n * (N_BINS + 1) * self.N * 8
        return out, [device.info_dict(r) for r in info]


def solve_with_fct(fb: "device.FactorBatch", mets: Sequence["device.MetDevice"], E: torch.Tensor,
                   passes: int, tol: float, maxiter: int = 200, dtau: float = DTAU):
    """Deferred FCT correction on already factored orbits (the forward driver's
    schedule, orbit/cli.py:1204-1241): pass 0 without FCT, then ``passes``
    solves whose right-hand side adds the limited anti-diffusive source of the
    previous pass's end-of-bin concentrations, warm-started from the previous
    c_0.  All orbits of the batch and all bins run on the device (K2 per bin
    over every orbit at once).  Returns the final orbits and a list of the
    per-pass info arrays."""
    orb, info = fb.solve(E, tol=tol, maxiter=maxiter, dtau=dtau)
    infos = [info]
    n = E.shape[0]
    for _ in range(passes):
        d = torch.stack([device.fct_source(mets[t], orb[:, t + 1].contiguous(), dtau) for t in range(N_BINS)],
                        dim=1)  # (n, 8, N)
        orb, info = fb.solve(E + d, c_warm=orb[:, 0].contiguous(), tol=tol, maxiter=maxiter, dtau=dtau)
        infos.append(info)
    return orb, infos


def solve_shared_operator(sym: Symbolic, T_stencils: Sequence[torch.Tensor], sinks: Sequence[torch.Tensor],
                          forcing: torch.Tensor, adjoint: bool = False, precision: int = 32,
                          tol: float = 1e-6, maxiter: int = 200, dtau: float = DTAU):
    """Many right-hand sides on one operator (marginal emission perturbations, or
    adjoint receptors with the transposed chain): one factor set of 8 bins,
    every solve slot mapped onto it, all orbits in one batched GMRES."""
    n = forcing.shape[0]
    fb = device.FactorBatch(sym, n, precision, n_sets=1)
    fb.numeric(list(T_stencils), list(sinks), dtau)
    if adjoint:
        return fb.solve_adjoint(forcing, tol=tol, maxiter=maxiter)
    return fb.solve(forcing, tol=tol, maxiter=maxiter, dtau=dtau)
