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
                 leaf_cells: int = 0, sym: Optional[Symbolic] = None, periodic: bool = False):
        self.sym = sym if sym is not None else Symbolic(nz, ny, nx, leaf_cells, periodic=periodic)
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


def fct_operators(mets: Sequence["device.MetDevice"], c_base: torch.Tensor, dtau: float = DTAU) -> torch.Tensor:
    """Frozen-gain L_AD of every bin at the baseline orbits' end-of-bin
    concentrations (the marginal convention, marginal.py:627-635): (n, 8, 7, N)."""
    n, N = c_base.shape[0], c_base.shape[-1]
    L = torch.empty((n, N_BINS, 7, N), dtype=torch.float64, device=c_base.device)
    for t in range(N_BINS):
        L[:, t] = device.fct_linear_operator(mets[t], c_base[:, t + 1].contiguous(), dtau).reshape(n, 7, N)
    return L


def _outer_gmres(g_of, b: torch.Tensor, rel_tol: float, max_iters: int):
    """Restarted GMRES (modified Gram-Schmidt, Givens) on (I - K) x = b for the
    affine map g(x) = K x + b, x0 = b, atol = 0.3 rel_tol ||b||, restart
    min(max_iters, 30) -- the outer solver of the marginal and adjoint FCT
    corrections (marginal.py:697-720, adjoint.py:868-941).  Every application
    of K is one batched device solve.  Returns (x, iterations, converged)."""
    bnorm = float(torch.linalg.norm(b))
    atol = 0.3 * rel_tol * bnorm
    restart = min(max_iters, 30)

    def matvec(v):
        return v - (g_of(v) - b)

    x = b.clone()
    iters, converged = 0, bnorm == 0.0
    while not converged and iters < max_iters:
        r = b - matvec(x)
        beta = float(torch.linalg.norm(r))
        if beta <= atol:
            converged = True
            break
        V = [r / beta]
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        gvec = np.zeros(restart + 1)
        gvec[0] = beta
        j = 0
        for j in range(min(restart, max_iters - iters)):
            w = matvec(V[j])
            for i in range(j + 1):  # modified Gram-Schmidt
                H[i, j] = float(torch.dot(w, V[i]))
                w = w - H[i, j] * V[i]
            H[j + 1, j] = float(torch.linalg.norm(w))
            V.append(w / H[j + 1, j] if H[j + 1, j] > 0 else w)
            for i in range(j):
                t0 = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t0
            den = np.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = (H[j, j] / den, H[j + 1, j] / den) if den > 0 else (1.0, 0.0)
            H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
            H[j + 1, j] = 0.0
            gvec[j + 1] = -sn[j] * gvec[j]
            gvec[j] = cs[j] * gvec[j]
            iters += 1
            if abs(gvec[j + 1]) <= atol:
                break
        k = j + 1
        y = np.linalg.solve(np.triu(H[:k, :k]), gvec[:k])
        for i in range(k):
            x = x + float(y[i]) * V[i]
        if abs(gvec[k]) <= atol:
            converged = True
    return x, iters, converged


def solve_marginal_fct(fb: "device.FactorBatch", mets: Sequence["device.MetDevice"], L_AD: torch.Tensor,
                       E: torch.Tensor, tol: float = 1e-6, rel_tol: float = 2e-3, max_iters: int = 40,
                       maxiter: int = 200, dtau: float = DTAU):
    """Marginal FCT outer solve (marginal.py:627-720) for a batch of orbits on
    the device.  The deferred correction delta_c = K delta_c + b (b the orbit of
    the forcing E, K v the orbit of the extra right-hand sides
    -L_AD[o][tau] v[o][tau+1]) is solved as restarted GMRES on (I - K) delta_c
    = b over the whole batch (x0 = b, atol = 0.3 rel_tol ||b||, restart
    min(max_iters, 30)); every application of K is one batched device solve of
    all orbits.  A last pass at the solution returns consistent orbits.
    Returns (orbits (n, 9, N), info dict)."""
    n, N = E.shape[0], E.shape[-1]
    g0 = mets[0]
    nz, ny, nx = g0.nz, g0.ny, g0.nx
    solves = [0]

    def inner(extra):
        orb, _ = fb.solve(E if extra is None else E + extra, tol=tol, maxiter=maxiter, dtau=dtau)
        solves[0] += 1
        return orb.reshape(-1)

    def extra_of(v):
        vv = v.reshape(n, N_BINS + 1, N)
        ex = torch.empty((n, N_BINS, N), dtype=torch.float64, device=E.device)
        for t in range(N_BINS):
            ex[:, t] = device.stencil_apply(nz, ny, nx, L_AD[:, t], vv[:, t + 1].contiguous(), alpha=-1.0)
        return ex

    b = inner(None)
    x, iters, converged = _outer_gmres(lambda v: inner(extra_of(v)), b, rel_tol, max_iters)
    g = inner(extra_of(x))
    rel_final = float((g - x).abs().max() / max(float(g.abs().max()), 1e-30))
    info = {"outer_iters": iters, "inner_solves": solves[0], "rel_final": rel_final, "converged": converged}
    return g.reshape(n, N_BINS + 1, N), info


def solve_adjoint_fct(fb: "device.FactorBatch", mets: Sequence["device.MetDevice"], L_AD: torch.Tensor,
                      R: torch.Tensor, tol: float = 1e-6, rel_tol: float = 2e-3, max_iters: int = 40,
                      maxiter: int = 200, dtau: float = DTAU):
    """Adjoint FCT outer solve (adjoint.py:521-566, 814-960) for a batch of
    receptor sets on the device.  L_low^T stays the factored propagator; the
    transposed anti-diffusive term enters as a deferred receptor.  The
    co-forcing mu_tau = lambda_tau - R_tau (R the effective receptor) solves
    the affine fixed point mu = K mu + b: b is the low-order adjoint's mu, K mu
    the mu of the adjoint solve whose receptor adds
    nu_sigma = -dtau L_AD[sigma-1]^T mu[sigma-1] (bins mod 8; L_AD[tau] frozen
    at the baseline's end-of-bin c[tau+1], the stencils of ``fct_operators``).
    Restarted GMRES on (I - K) mu = b over the whole batch, every application
    of K one batched transposed device solve, then a final pass at the
    solution.  Returns (adjoint orbits (n, 9, N), effective receptors
    (n, 8, N), info dict); dJ/de_tau = dtau (lambda_tau - R_tau) holds for them."""
    n, N = R.shape[0], R.shape[-1]
    g0 = mets[0]
    nz, ny, nx = g0.nz, g0.ny, g0.nx
    solves = [0]

    def inner(nu):
        Reff = R if nu is None else R + nu
        lam, _ = fb.solve_adjoint(Reff, tol=tol, maxiter=maxiter)
        solves[0] += 1
        return (lam[:, :N_BINS] - Reff).reshape(-1), lam, Reff

    def recep_of(mu):
        mm = mu.reshape(n, N_BINS, N)
        nu = torch.empty((n, N_BINS, N), dtype=torch.float64, device=R.device)
        for t in range(N_BINS):
            src = (t - 1) % N_BINS
            nu[:, t] = device.stencil_apply(nz, ny, nx, L_AD[:, src], mm[:, src].contiguous(), alpha=-dtau,
                                            trans=True)
        return nu

    b, _, _ = inner(None)
    x, iters, converged = _outer_gmres(lambda v: inner(recep_of(v))[0], b, rel_tol, max_iters)
    g, lam, Reff = inner(recep_of(x))
    rel_final = float((g - x).abs().max() / max(float(g.abs().max()), 1e-30))
    info = {"outer_iters": iters, "inner_solves": solves[0], "rel_final": rel_final, "converged": converged}
    return lam, Reff, info
