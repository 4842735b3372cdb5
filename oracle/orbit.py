"""Oracle: SuperLU periodic-orbit GMRES solve, forward and adjoint.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates the
reference's documented no-UMFPACK path (SciPy SuperLU, COLAMD):

* ``_factor_one_bin`` (``umfpack_sym=None``)  orbit/core/orbit.py:79-96,
                                              orbit/core/solve.py:361-365
* ``apply_monodromy``                         orbit/core/orbit.py:99-107
* ``compute_s``                               orbit/core/orbit.py:110-120
* ``solve_orbit_one_species``                 orbit/core/orbit.py:123-210
* ``apply_monodromy_adjoint``                 orbit/core/orbit_adjoint.py:36-47
* ``compute_s_adjoint``                       orbit/core/orbit_adjoint.py:50-67
* ``solve_orbit_adjoint_one_species``         orbit/core/orbit_adjoint.py:70-144
* ``gradient_per_emission_bin``               orbit/core/orbit_adjoint.py:147-153
* the FCT deferred-correction schedule        orbit/cli.py:1204-1241
* the marginal FCT outer GMRES                orbit/modes/marginal.py:627-720
* the adjoint FCT outer GMRES                 orbit/modes/adjoint.py:521-566, 814-960
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

DTAU = 10800.0
N_BINS = 8


def factor_one_bin(L, dtau=DTAU):
    """A = I + dtau L, CSC, duplicates summed, indices sorted, then splu."""
    N = L.shape[0]
    A = (sp.eye(N, format="csc") + L * dtau).tocsc()
    A.sum_duplicates()
    A.sort_indices()
    return spla.splu(A)


def apply_monodromy(v, lus):
    x = np.array(v, dtype=np.float64, copy=True)
    for tau in range(N_BINS):
        x = lus[tau].solve(x)
    return x


def compute_s(lus, e_list, dtau=DTAU):
    x = np.zeros(lus[0].shape[0])
    for tau in range(N_BINS):
        x = lus[tau].solve(x + dtau * e_list[tau])
    return x


def solve_orbit_one_species(lus, e_list, dtau=DTAU, c_warm=None, tol=1e-6, maxiter=200):
    """GMRES(30) on (I - M) c0 = s with atol = tol ||s||; orbit recovery and
    diagnostics as in orbit.py:123-210."""
    N = lus[0].shape[0]
    s = compute_s(lus, e_list, dtau)
    sn = np.linalg.norm(s)
    if sn < 1e-30:
        z = np.zeros(N)
        return [z.copy() for _ in range(N_BINS + 1)], dict(
            gmres_iters=0, residual=0.0, periodicity=0.0, neg_frac=0.0)
    op = spla.LinearOperator((N, N), matvec=lambda v: v - apply_monodromy(v, lus),
                             dtype=np.float64)
    x0 = c_warm if c_warm is not None else s.copy()
    it = [0]

    def cb(_):
        it[0] += 1

    c0, code = spla.gmres(op, s, x0=x0, rtol=1e-30, atol=tol * sn, restart=30,
                          maxiter=maxiter, callback=cb, callback_type="pr_norm")
    orbit = [c0.copy()]
    x = c0.copy()
    for tau in range(N_BINS):
        x = lus[tau].solve(x + dtau * e_list[tau])
        orbit.append(x.copy())
    res = np.linalg.norm(op.matvec(c0) - s) / sn
    per = np.linalg.norm(orbit[-1] - c0) / (np.linalg.norm(c0) + 1e-30)
    neg = float(np.mean(np.concatenate(orbit) < 0))
    return orbit, dict(gmres_iters=it[0], residual=float(res), periodicity=float(per),
                       neg_frac=neg, converged=(code == 0))


def apply_monodromy_adjoint(v, lus):
    x = np.array(v, dtype=np.float64, copy=True)
    for tau in range(N_BINS - 1, -1, -1):
        x = lus[tau].solve(x, trans="T")
    return x


def compute_s_adjoint(lus, R_list):
    x = np.zeros(lus[0].shape[0])
    for tau in range(N_BINS - 1, -1, -1):
        x = lus[tau].solve(x, trans="T") + R_list[tau]
    return x


def solve_orbit_adjoint_one_species(lus, R_list, lam_warm=None, tol=1e-6, maxiter=200):
    N = lus[0].shape[0]
    s = compute_s_adjoint(lus, R_list)
    sn = np.linalg.norm(s)
    if sn < 1e-30:
        z = np.zeros(N)
        return [z.copy() for _ in range(N_BINS + 1)], dict(gmres_iters=0, residual=0.0,
                                                           periodicity=0.0)
    op = spla.LinearOperator((N, N), matvec=lambda v: v - apply_monodromy_adjoint(v, lus),
                             dtype=np.float64)
    x0 = lam_warm if lam_warm is not None else s.copy()
    it = [0]

    def cb(_):
        it[0] += 1

    lam0, code = spla.gmres(op, s, x0=x0, rtol=1e-30, atol=tol * sn, restart=30,
                            maxiter=maxiter, callback=cb, callback_type="pr_norm")
    adj = [None] * (N_BINS + 1)
    adj[0] = lam0.copy()
    adj[N_BINS] = lam0.copy()
    x = lam0.copy()
    for tau in range(N_BINS - 1, 0, -1):
        x = lus[tau].solve(x, trans="T") + R_list[tau]
        adj[tau] = x.copy()
    res = np.linalg.norm(op.matvec(lam0) - s) / sn
    chk = lus[0].solve(adj[1], trans="T") + R_list[0]
    per = np.linalg.norm(chk - lam0) / (np.linalg.norm(lam0) + 1e-30)
    return adj, dict(gmres_iters=it[0], residual=float(res), periodicity=float(per),
                     converged=(code == 0))


def gradient_per_emission_bin(adjoint, R_list, dtau=DTAU):
    return [dtau * (adjoint[t] - R_list[t]) for t in range(N_BINS)]


def fct_deferred_solve(lus, e_list, met, passes, tol=1e-8, maxiter=200, dtau=DTAU):
    """Pass 0 without FCT, then ``passes`` solves whose RHS adds the FCT source
    of the previous pass's end-of-bin concentrations (cli.py:1204-1241); the
    previous pass's c_0 warm-starts the next (cli.py:2382-2392 uses the
    previous iterate)."""
    from oracle.fct import fct_source
    orbit, info = solve_orbit_one_species(lus, e_list, dtau, None, tol, maxiter)
    infos = [info]
    for _ in range(passes):
        rhs = [e_list[t] + fct_source(met[t], orbit[t + 1], dtau) for t in range(N_BINS)]
        orbit, info = solve_orbit_one_species(lus, rhs, dtau, orbit[0], tol, maxiter)
        infos.append(info)
    return orbit, infos


def fct_outer_solve(lus_per_orbit, e_lists, L_AD, tol=1e-8, rel_tol=2e-3, max_iters=40, dtau=DTAU):
    """Marginal FCT outer solve (orbit/modes/marginal.py:627-720): the deferred
    correction delta_c = K delta_c + b, b the low-order solution of the forcing,
    K v the orbit of the extra right-hand sides -L_AD[o][tau] v[o][tau+1], solved
    as GMRES on (I - K) delta_c = b over all orbits flattened (x0 = b,
    atol = 0.3 rel_tol ||b||, restart min(max_iters, 30)), then one final pass
    at the solution.  Returns (orbits per orbit as 9 arrays, outer iterations,
    rel_final = max|g(x) - x| / max|g(x)|)."""
    n = len(lus_per_orbit)
    N = lus_per_orbit[0][0].shape[0]

    def inner(extra):
        out = []
        for o in range(n):
            e = [e_lists[o][t] + (extra[o][t] if extra is not None else 0.0) for t in range(N_BINS)]
            orb, _ = solve_orbit_one_species(lus_per_orbit[o], e, dtau=dtau, tol=tol)
            out.append(np.concatenate(orb))
        return np.concatenate(out)

    def extra_of(v):
        vv = v.reshape(n, N_BINS + 1, N)
        return [[-(L_AD[o][t] @ vv[o][t + 1]) for t in range(N_BINS)] for o in range(n)]

    b = inner(None)
    op = spla.LinearOperator((b.size, b.size), matvec=lambda v: v - (inner(extra_of(v)) - b), dtype=np.float64)
    restart = min(max_iters, 30)
    hist = []
    x, _ = spla.gmres(op, b, x0=b.copy(), rtol=1e-30, atol=0.3 * rel_tol * np.linalg.norm(b), restart=restart,
                      maxiter=max(1, -(-max_iters // restart)), callback=lambda r: hist.append(r),
                      callback_type="pr_norm")
    g = inner(extra_of(x))
    rel = float(np.abs(g - x).max() / max(np.abs(g).max(), 1e-30))
    orbits = [list(v) for v in g.reshape(n, N_BINS + 1, N)]
    return orbits, len(hist), rel


def fct_adjoint_outer_solve(lus_per_orbit, R_lists, L_AD, tol=1e-8, rel_tol=2e-3, max_iters=40, dtau=DTAU):
    """Adjoint FCT outer solve (orbit/modes/adjoint.py:521-566, 814-960): L_low^T
    stays the factored propagator and the transposed anti-diffusive term enters
    as a deferred receptor.  The co-forcing mu_tau = lambda_tau - R_tau (R the
    effective receptor) satisfies the affine fixed point mu = K mu + b: b is the
    low-order adjoint's mu, and K mu the mu of the adjoint solve whose receptor
    adds nu_sigma = -dtau L_AD[sigma-1]^T mu[sigma-1] (bins mod 8; L_AD[tau]
    frozen at the baseline's end-of-bin c[tau+1]).  Solved as GMRES on
    (I - K) mu = b over all orbits flattened (x0 = b, atol = 0.3 rel_tol ||b||,
    restart min(max_iters, 30)), then one final pass at the solution.  Returns
    (adjoint orbits per orbit as 9 arrays, effective receptors per orbit as 8
    arrays, outer iterations, rel_final = max|g(x) - x| / max|g(x)|)."""
    n = len(lus_per_orbit)
    N = lus_per_orbit[0][0].shape[0]

    def recep_of(mu):
        mm = mu.reshape(n, N_BINS, N)
        return [[-dtau * (L_AD[o][(t - 1) % N_BINS].T @ mm[o][(t - 1) % N_BINS]) for t in range(N_BINS)]
                for o in range(n)]

    def inner(extra):
        mus, lams, Rs = [], [], []
        for o in range(n):
            R = [R_lists[o][t] + (extra[o][t] if extra is not None else 0.0) for t in range(N_BINS)]
            lam, _ = solve_orbit_adjoint_one_species(lus_per_orbit[o], R, tol=tol)
            mus.append(np.concatenate([lam[t] - R[t] for t in range(N_BINS)]))
            lams.append(lam)
            Rs.append(R)
        return np.concatenate(mus), lams, Rs

    b, _, _ = inner(None)
    op = spla.LinearOperator((b.size, b.size), matvec=lambda v: v - (inner(recep_of(v))[0] - b),
                             dtype=np.float64)
    restart = min(max_iters, 30)
    hist = []
    x, _ = spla.gmres(op, b, x0=b.copy(), rtol=1e-30, atol=0.3 * rel_tol * np.linalg.norm(b), restart=restart,
                      maxiter=max(1, -(-max_iters // restart)), callback=lambda r: hist.append(r),
                      callback_type="pr_norm")
    g, lams, Rs = inner(recep_of(x))
    rel = float(np.abs(g - x).max() / max(np.abs(g).max(), 1e-30))
    return lams, Rs, len(hist), rel
