"""Parity on the 80x72x15 benchmark workload itself (B200).

The benchmark's first met draw (86,400 cells, convective mass flux in 30 % of
the columns) and its species 0 and 1, with the analysis the benchmark runs
(the autotuner's entry: nested-dissection leaf 80, tensor-core supernodes
from n = 32).  The truth is the reference's own orbit at tol 1e-12 (SciPy
SuperLU, its no-UMFPACK path), committed as a digest by
tests/golden/make_bench_golden.py: values at 16,384 fixed random (bin, cell)
positions plus every bin's max |c| and L2 norm.

* FP64 drop-in at tol 1e-10: max |c - c_ref| / max |c_ref| over the sampled
  positions <= 1e-8, every bin's max and norm within 1e-8;
* mixed precision (FP32 factors, FP64 refinement) at the benchmark's tol 1e-8:
  the same measures <= 1e-6;
* both orbits satisfy the eight FP64 bin equations A_tau c_{tau+1} = c_tau +
  dtau e_tau over every cell (a size-independent check of the whole orbit);
* the mass-balance statistics of the eight bins equal the reference's and the
  gate decision (interior p90 > 0.05 per day aborts) is the same.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DIGEST = os.path.join(HERE, "golden", "bench_grid_digest.npz")
NZ, NY, NX = 15, 72, 80
SEED = 2024
DTAU = 10800.0


@pytest.fixture(scope="module")
def work():
    import torch
    from orbit_b200 import device, synthetic
    from orbit_b200.shard import met_draw_seed
    from orbit_b200.symbolic import Symbolic
    z = dict(np.load(DIGEST))
    species = [int(s) for s in z["species"]]
    met = synthetic.make_met(met_draw_seed(SEED, 0, 0), NZ, NY, NX, cmfmc_frac=0.3)
    spc = [synthetic.make_species(SEED + 17 + s, NZ, NY, NX) for s in range(max(species) + 1)]
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(spc[s].sink_diag(met), device="cuda") for s in species]
    E = torch.as_tensor(np.stack([spc[s].emis for s in species]), device="cuda")
    sym = Symbolic.tuned(NZ, NY, NX, 32, 12)
    out = {}
    for prec, tol in ((64, 1e-10), (32, 1e-8)):
        fb = device.FactorBatch(sym, len(species), prec)
        fb.numeric([T[t] for _ in species for t in range(8)], [sinks[k][t] for k in range(len(species))
                                                              for t in range(8)])
        orb, info = fb.solve(E, tol=tol)
        out[prec] = (orb, info)
        fb.close()
    return z, species, mets, T, sinks, E, out


def _digest_errors(z, s, orb):
    C = orb.cpu().numpy()
    ref_max = z[f"s{s}_max"]
    err_pts = np.abs(C.reshape(-1)[z["pos"]] - z[f"s{s}_vals"]).max() / ref_max.max()
    err_max = np.abs(np.abs(C).max(axis=1) - ref_max).max() / ref_max.max()
    err_norm = (np.abs(np.linalg.norm(C, axis=1) - z[f"s{s}_norm"]) / z[f"s{s}_norm"]).max()
    return err_pts, err_max, err_norm


def _bin_equation_residual(T, sink, e, orb):
    """max over bins of ||A_tau c_{tau+1} - c_tau - dtau e_tau|| / ||c_tau + dtau e_tau||,
    A_tau = I + dtau (T_tau + diag d_tau), all in FP64 on the device."""
    import torch
    from orbit_b200 import device
    worst = 0.0
    for t in range(8):
        c1 = orb[t + 1].contiguous()
        Ac = c1 + DTAU * (device.stencil_apply(NZ, NY, NX, T[t], c1) + sink[t] * c1)
        rhs = orb[t] + DTAU * e[t]
        worst = max(worst, float(torch.linalg.norm(Ac - rhs) / torch.linalg.norm(rhs)))
    return worst


@pytest.mark.parametrize("prec,bound", [(64, 1e-8), (32, 1e-6)])
def test_bench_orbits_match_reference(work, prec, bound):
    z, species, mets, T, sinks, E, out = work
    orb, info = out[prec]
    assert np.all(info[:, 4] > 0), info
    for k, s in enumerate(species):
        e_pts, e_max, e_norm = _digest_errors(z, s, orb[k])
        assert e_pts <= bound, (prec, s, e_pts)
        assert e_max <= bound, (prec, s, e_max)
        assert e_norm <= bound, (prec, s, e_norm)
        assert _bin_equation_residual(T, sinks[k], E[k], orb[k]) <= (1e-9 if prec == 64 else 1e-7)


def test_bench_mass_balance_gate_matches_reference(work):
    from orbit_b200 import device
    z, species, mets, T, sinks, E, out = work
    mb = device.mass_balance(mets, T)
    got = np.array([mb[str(k)] for k in z["mb_keys"]])
    np.testing.assert_allclose(got, z["mb_vals"], rtol=1e-9, atol=1e-12)
    assert (mb["interior_p90"] > 0.05) == (z["mb_vals"][1] > 0.05)
