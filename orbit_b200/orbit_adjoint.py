"""Drop-in for the reference's periodic-orbit adjoint (orbit/core/orbit_adjoint.py).

``apply_monodromy_adjoint`` (orbit_adjoint.py:36-47) and ``compute_s_adjoint``
(:50-67) run the transposed chain P_0^T ... P_7^T as one device launch;
``solve_orbit_adjoint_one_species`` (:70-144) runs GMRES on
(I - M^T) lambda_0 = s_adj on the device and unrolls the adjoint orbit;
``gradient_per_emission_bin`` (:147-153) is the same host identity.  The
LU list is the forward one (DeviceLUs), read transposed.
"""
from __future__ import annotations

import numpy as np

from .orbit import _bin_set
from .synthetic import DTAU, N_BINS


def apply_monodromy_adjoint(v, lu_list_8):
    import torch
    bs = _bin_set(lu_list_8)
    x = torch.as_tensor(np.ascontiguousarray(v, dtype=np.float64), device="cuda")[None]
    return bs.fb.chain(x, trans=True)[0].cpu().numpy()


def compute_s_adjoint(lu_list_8, R_list):
    import torch
    bs = _bin_set(lu_list_8)
    R = torch.as_tensor(np.stack([np.asarray(r, dtype=np.float64) for r in R_list]), device="cuda")
    x = torch.zeros((1, bs.N), dtype=torch.float64, device="cuda")
    return bs.fb.chain(x, trans=True, forcing=R[None], fscale=1.0)[0].cpu().numpy()


def solve_orbit_adjoint_one_species(lu_list_8, R_list, *, lam_warm=None, tol=1e-6, maxiter=200):
    import torch
    bs = _bin_set(lu_list_8)
    R = torch.as_tensor(np.stack([np.asarray(r, dtype=np.float64) for r in R_list]), device="cuda")
    w = None if lam_warm is None else torch.as_tensor(np.asarray(lam_warm, dtype=np.float64), device="cuda")
    adj, info = bs.fb.solve_adjoint(R[None], lam_warm=w, tol=tol, maxiter=maxiter)
    a = adj[0].cpu().numpy()
    return [a[t].copy() for t in range(N_BINS + 1)], dict(
        gmres_iters=int(info[0, 0]), residual=float(info[0, 1]), periodicity=float(info[0, 2]))


def gradient_per_emission_bin(adjoint, R_list):
    return [DTAU * (adjoint[tau] - R_list[tau]) for tau in range(N_BINS)]
