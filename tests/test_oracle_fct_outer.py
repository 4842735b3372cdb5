"""The oracle's marginal and adjoint FCT outer solves (restating
orbit/modes/marginal.py:627-720 and orbit/modes/adjoint.py:521-566, 814-960),
pinned on the CPU on a tiny grid.

The deferred correction delta_c = K delta_c + b is linear: b is the orbit of
the perturbation's forcing, K v the orbit of the extra right-hand sides
-L_AD[tau] v[tau + 1].  Built column by column, (I - K) x = b can be solved
densely; the oracle's GMRES result must match it, satisfy the fixed point to
its tolerance, and reduce to the plain orbit solve when L_AD vanishes.
"""
import numpy as np
import scipy.sparse as sp

from oracle import assembly, fct as ofct, orbit as oorbit
from orbit_b200 import synthetic

NZ, NY, NX = 3, 4, 5
N = NZ * NY * NX


def _setup():
    met = synthetic.make_met(9, NZ, NY, NX, cmfmc_frac=0.3)
    spc = synthetic.make_species(31, NZ, NY, NX)
    d = spc.sink_diag(met)
    lus = [oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(met[t]), d[t]))
           for t in range(8)]
    base, _ = oorbit.solve_orbit_one_species(lus, list(spc.emis), tol=1e-13)
    LAD = [ofct.fct_linear_operator(met[t], np.asarray(base[t + 1]), 10800.0) for t in range(8)]
    dE = np.zeros_like(np.asarray(spc.emis))
    dE[:, : NY * NX] = 0.1 * np.asarray(spc.emis)[:, : NY * NX]  # perturbed surface layer
    return lus, LAD, dE


def _orbit(lus, forcing):
    orb, _ = oorbit.solve_orbit_one_species(lus, forcing, tol=1e-14)
    return np.concatenate([np.asarray(o) for o in orb])


def test_outer_solve_matches_dense_fixed_point():
    lus, LAD, dE = _setup()
    orbs, iters, rel = oorbit.fct_outer_solve([lus], [list(dE)], [LAD], tol=1e-14, rel_tol=1e-11, max_iters=60)
    x = np.concatenate([np.asarray(o) for o in orbs[0]])
    assert rel < 1e-8 and iters > 0
    b = _orbit(lus, list(dE))

    def K(v):
        vv = v.reshape(9, N)
        return _orbit(lus, [-(LAD[t] @ vv[t + 1]) for t in range(8)])

    n = b.size
    Km = np.stack([K(np.eye(n)[:, j]) for j in range(n)], axis=1)
    xd = np.linalg.solve(np.eye(n) - Km, b)
    assert np.abs(x - xd).max() <= 1e-7 * np.abs(xd).max()


def test_outer_solve_without_coupling_is_the_plain_orbit():
    lus, LAD, dE = _setup()
    zero = [sp.csc_matrix((N, N)) for _ in range(8)]
    orbs, _, rel = oorbit.fct_outer_solve([lus], [list(dE)], [zero], tol=1e-14, rel_tol=1e-10)
    x = np.concatenate([np.asarray(o) for o in orbs[0]])
    want = _orbit(lus, list(dE))
    assert np.abs(x - want).max() <= 1e-10 * np.abs(want).max()
    assert rel < 1e-10


def _adjoint_mu(lus, R):
    lam, _ = oorbit.solve_orbit_adjoint_one_species(lus, R, tol=1e-14)
    return np.concatenate([np.asarray(lam[t]) - R[t] for t in range(8)])


def test_adjoint_outer_solve_matches_dense_fixed_point():
    """mu = K mu + b with K mu the co-forcing of the adjoint solve whose receptor
    adds -dtau L_AD[sigma-1]^T mu[sigma-1]: the oracle's GMRES equals the dense
    solution of (I - K) mu = b, and its final pass is consistent."""
    lus, LAD, _ = _setup()
    rng = np.random.default_rng(2)
    R = [rng.random(N) * (t + 1) for t in range(8)]
    lams, Rs, iters, rel = oorbit.fct_adjoint_outer_solve([lus], [R], [LAD], tol=1e-14, rel_tol=1e-11,
                                                         max_iters=60)
    assert rel < 1e-8 and iters > 0
    mu = np.concatenate([np.asarray(lams[0][t]) - Rs[0][t] for t in range(8)])
    b = _adjoint_mu(lus, R)

    def K(v):
        vv = v.reshape(8, N)
        nu = [R[t] - 10800.0 * (LAD[(t - 1) % 8].T @ vv[(t - 1) % 8]) for t in range(8)]
        return _adjoint_mu(lus, nu) - b

    n = b.size
    Km = np.stack([K(np.eye(n)[:, j]) for j in range(n)], axis=1)
    xd = np.linalg.solve(np.eye(n) - Km, b)
    assert np.abs(mu - xd).max() <= 1e-7 * np.abs(xd).max()


def test_adjoint_outer_solve_without_coupling_is_the_plain_adjoint():
    lus, _, _ = _setup()
    zero = [sp.csc_matrix((N, N)) for _ in range(8)]
    rng = np.random.default_rng(3)
    R = [rng.random(N) for _ in range(8)]
    lams, Rs, _, rel = oorbit.fct_adjoint_outer_solve([lus], [R], [zero], tol=1e-14, rel_tol=1e-10)
    want, _ = oorbit.solve_orbit_adjoint_one_species(lus, R, tol=1e-14)
    got = np.stack([np.asarray(v) for v in lams[0]])
    want = np.stack([np.asarray(v) for v in want])
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    assert rel < 1e-10
