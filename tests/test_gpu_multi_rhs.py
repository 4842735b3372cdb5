"""Many right-hand sides on one factor set (B200).

Marginal perturbations and adjoint receptors of one operator share a single
factor set (the reference reuses one lu_list_8 for all receptors,
orbit/modes/adjoint.py:573-583).  When every solve slot maps onto one set,
the chained solves serve groups of right-hand sides per task (forward: the
staged kernel with K vectors; transposed: the column-oriented kernel with K
vectors).  Solving 64 receptors (or 64 perturbations) in one call must give
the same orbits as solving each alone, to 1e-10 relative in FP64 and to the
1e-6 mixed-precision bar with FP32 factors.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NZ, NY, NX = 6, 10, 12
N_RHS = 64


def _setup(precision):
    import torch
    from orbit_b200 import device, synthetic
    from orbit_b200.symbolic import Symbolic
    met = synthetic.make_met(77, NZ, NY, NX, cmfmc_frac=0.3)
    spc = synthetic.make_species(78, NZ, NY, NX)
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(d, device="cuda") for d in spc.sink_diag(met)]
    sym = Symbolic(NZ, NY, NX, 16)
    rng = np.random.default_rng(5)
    N = NZ * NY * NX
    F = np.zeros((N_RHS, 8, N))
    for q in range(N_RHS):
        j0, i0 = rng.integers(0, NY - 3), rng.integers(0, NX - 3)
        f = np.zeros((8, NZ, NY, NX))
        f[:, 0, j0:j0 + 3, i0:i0 + 3] = rng.random((8, 3, 3))
        F[q] = f.reshape(8, N)
    return device, sym, T, sinks, torch.as_tensor(F, device="cuda")


@pytest.mark.parametrize("precision,bound", [(64, 1e-10), (32, 1e-6)])
@pytest.mark.parametrize("adjoint", [False, True])
def test_many_rhs_equal_one_at_a_time(precision, bound, adjoint):
    device, sym, T, sinks, F = _setup(precision)
    tol = 1e-12 if precision == 64 else 1e-9
    fb = device.FactorBatch(sym, N_RHS, precision, n_sets=1)
    fb.numeric(T, sinks)
    one = device.FactorBatch(sym, 1, precision, n_sets=1)
    one.numeric(T, sinks)
    if adjoint:
        many, info = fb.solve_adjoint(F * 1e-3, tol=tol)
    else:
        many, info = fb.solve(F * 1e-9, tol=tol)
    assert np.all(info[:, 4] > 0)
    many = many.cpu().numpy()
    for q in range(0, N_RHS, 7):
        if adjoint:
            o1, _ = one.solve_adjoint(F[q:q + 1] * 1e-3, tol=tol)
        else:
            o1, _ = one.solve(F[q:q + 1] * 1e-9, tol=tol)
        ref = o1[0].cpu().numpy()
        err = np.abs(many[q] - ref).max() / np.abs(ref).max()
        assert err <= bound, (q, err)
