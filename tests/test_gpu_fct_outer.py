"""Marginal FCT outer solve on the device against the oracle (B200).

On a small grid (6x8x10, two species, FP64 factors) the device driver
(batched inner orbit solves, L_AD and its products on the device, GMRES on
(I - K) delta_c = b over the batch) must reach the oracle's fixed point
(SuperLU inner solves, SciPy GMRES, the oracle's L_AD from the same baseline
orbits) to 1e-8 relative (the FP64 bar), with the final pass consistent with
the solution to 1e-8.
The transposed stencil product is checked against the explicit matrix.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NZ, NY, NX = 6, 8, 10


def test_stencil_apply_and_transpose():
    import torch
    from orbit_b200 import device
    rng = np.random.default_rng(3)
    N = NZ * NY * NX
    S = rng.standard_normal((2, 7, N))
    x = rng.standard_normal((2, N))
    St, xt = torch.as_tensor(S, device="cuda"), torch.as_tensor(x, device="cuda")
    y = device.stencil_apply(NZ, NY, NX, St, xt, alpha=-2.0).cpu().numpy()
    yt = device.stencil_apply(NZ, NY, NX, St, xt, trans=True).cpu().numpy()
    for v in range(2):
        A = device.stencil_to_csr(S[v], NZ, NY, NX)
        np.testing.assert_allclose(y[v], -2.0 * (A @ x[v]), rtol=1e-13, atol=1e-12)
        np.testing.assert_allclose(yt[v], A.T @ x[v], rtol=1e-13, atol=1e-12)


def test_marginal_fct_outer_matches_oracle():
    import torch
    from orbit_b200 import api, device, synthetic
    from orbit_b200.symbolic import Symbolic
    from oracle import assembly, fct as ofct, orbit as oorbit
    met = synthetic.make_met(31, NZ, NY, NX)
    spc = [synthetic.make_species(40 + k, NZ, NY, NX) for k in range(2)]
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    sym = Symbolic(NZ, NY, NX, 16)
    fb = device.FactorBatch(sym, 2, 64)
    sinks = [torch.as_tensor(d, device="cuda") for s in spc for d in s.sink_diag(met)]
    fb.numeric([T[t] for _ in range(2) for t in range(8)], sinks)
    E = torch.as_tensor(np.stack([s.emis for s in spc]), device="cuda")
    base, _ = fb.solve(E, tol=1e-12)
    L = api.fct_operators(mets, base)
    dE = torch.zeros_like(E)
    dE[:, :, : NY * NX // 2] = 0.1 * E[:, :, : NY * NX // 2]  # perturbation of half the surface layer
    orb, info = api.solve_marginal_fct(fb, mets, L, dE, tol=1e-12, rel_tol=1e-9, max_iters=60)
    assert info["converged"], info
    assert info["rel_final"] < 1e-8
    # oracle
    base_h, dE_h = base.cpu().numpy(), dE.cpu().numpy()
    lus, LAD = [], []
    for k, s in enumerate(spc):
        d = s.sink_diag(met)
        lus.append([oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(met[t]), d[t]))
                    for t in range(8)])
        LAD.append([ofct.fct_linear_operator(met[t], base_h[k, t + 1], 10800.0) for t in range(8)])
    orbs, _, rel = oorbit.fct_outer_solve(lus, [list(dE_h[k]) for k in range(2)], LAD, tol=1e-12, rel_tol=1e-9,
                                          max_iters=60)
    want = np.stack([np.stack(o) for o in orbs])
    got = orb.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()


def test_adjoint_fct_outer_matches_oracle():
    """Adjoint FCT outer solve (adjoint.py:521-566, 814-960) on the device against
    the oracle's restatement: two receptor sets on two species' operators, FP64
    factors, L_AD frozen at the baseline orbits; adjoint orbits and effective
    receptors within 1e-8 relative."""
    import torch
    from orbit_b200 import api, device, synthetic
    from orbit_b200.symbolic import Symbolic
    from oracle import assembly, fct as ofct, orbit as oorbit
    met = synthetic.make_met(31, NZ, NY, NX)
    spc = [synthetic.make_species(40 + k, NZ, NY, NX) for k in range(2)]
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    sym = Symbolic(NZ, NY, NX, 16)
    fb = device.FactorBatch(sym, 2, 64)
    sinks = [torch.as_tensor(d, device="cuda") for s in spc for d in s.sink_diag(met)]
    fb.numeric([T[t] for _ in range(2) for t in range(8)], sinks)
    E = torch.as_tensor(np.stack([s.emis for s in spc]), device="cuda")
    base, _ = fb.solve(E, tol=1e-12)
    L = api.fct_operators(mets, base)
    rng = np.random.default_rng(8)
    N = NZ * NY * NX
    R = np.zeros((2, 8, N))
    R[:, :, : NY * NX] = rng.random((2, 8, NY * NX))  # surface receptors
    lam, Reff, info = api.solve_adjoint_fct(fb, mets, L, torch.as_tensor(R, device="cuda"), tol=1e-12,
                                            rel_tol=1e-9, max_iters=60)
    assert info["converged"], info
    assert info["rel_final"] < 1e-8
    base_h = base.cpu().numpy()
    lus, LAD = [], []
    for k, s in enumerate(spc):
        d = s.sink_diag(met)
        lus.append([oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(met[t]), d[t]))
                    for t in range(8)])
        LAD.append([ofct.fct_linear_operator(met[t], base_h[k, t + 1], 10800.0) for t in range(8)])
    lams, Rs, _, _ = oorbit.fct_adjoint_outer_solve(lus, [list(R[k]) for k in range(2)], LAD, tol=1e-12,
                                                     rel_tol=1e-9, max_iters=60)
    want = np.stack([np.stack(x) for x in lams])
    got = lam.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()
    want_R = np.stack([np.stack(x) for x in Rs])
    assert np.abs(Reff.cpu().numpy() - want_R).max() <= 1e-8 * np.abs(want_R).max()
