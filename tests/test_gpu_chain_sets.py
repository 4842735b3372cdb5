"""Chained solves over shared and distinct factor sets (B200).

When every solve slot of a handle has its own factor set, the chained-solve
kernel streams the factor rows under an L2 evict-first policy; when slots
share a set (species slots of a serving batch, coupled species mapped onto
one operator) it keeps the normal policy, since the rows are reused from L2.
The policy is a cache hint only: four slots mapped onto two sets must give
bitwise the same chains, forward and transposed, as four slots with their own
copies of the same two factorizations.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NZ, NY, NX = 6, 10, 12


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("trans", [False, True])
def test_shared_sets_match_own_sets(precision, trans):
    import torch
    from orbit_b200 import device, synthetic
    from orbit_b200.symbolic import Symbolic
    met = synthetic.make_met(91, NZ, NY, NX, cmfmc_frac=0.3)
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    spc = [synthetic.make_species(92 + q, NZ, NY, NX) for q in range(2)]
    sinks = [[torch.as_tensor(d, device="cuda") for d in s.sink_diag(met)] for s in spc]
    sym = Symbolic(NZ, NY, NX, 16)
    shared = device.FactorBatch(sym, 4, precision, n_sets=2)
    shared.numeric(T + T, sinks[0] + sinks[1])
    shared.map([0, 1, 0, 1])
    own = device.FactorBatch(sym, 4, precision, n_sets=4)
    own.numeric(T * 4, sinks[0] + sinks[1] + sinks[0] + sinks[1])
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    x = torch.randn(4, sym.N, generator=g, device="cuda", dtype=torch.float64)
    a = shared.chain(x, trans=trans, refine=False).cpu().numpy()
    b = own.chain(x, trans=trans, refine=False).cpu().numpy()
    assert np.all(np.isfinite(a)) and np.abs(a).max() > 0
    assert np.array_equal(a, b)
    shared.close()
    own.close()
