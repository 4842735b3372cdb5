"""Drop-in entry points (reference names and signatures) on the device,
against the reference's golden vectors and the CPU oracle."""
import numpy as np
import pytest
import scipy.sparse as sp

import golden_io
from oracle import assembly, fct as ofct, orbit as oorbit

pytestmark = pytest.mark.gpu

Z = golden_io.load()
MET = golden_io.met_list(Z)
SPC = golden_io.species(Z)


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _L_list(scale_sink=1.0):
    d = SPC.sink_diag(MET)
    return [assembly.species_operator(assembly.transport_block(g), scale_sink * d[t]) for t, g in enumerate(MET)]


def test_lu_objects_and_orbit_dropin():
    from orbit_b200 import solve as osolve, orbit as oorb, orbit_adjoint as oadj
    L = _L_list()
    sym = osolve.umfpack_symbolic(L[0], verbose=False)
    assert sym["n"] == MET[0].N
    I_N = sp.eye(MET[0].N, format="csc")
    lus = [oorb._factor_one_bin(Lt, I_N, sym, None) for Lt in L]
    rng = np.random.default_rng(3)
    b = rng.standard_normal(MET[0].N)
    ref = oorbit.factor_one_bin(L[2])
    assert _rel(lus[2].solve(b), ref.solve(b)) < 1e-12
    assert _rel(lus[2].solve(b, trans="T"), ref.solve(b, trans="T")) < 1e-12
    assert _rel(oorb.apply_monodromy(Z["mono_v"], lus), Z["mono_Mv"]) < 1e-12
    # the bin-set factorization replaced lus[2]'s own: one set of factors per LU,
    # and .solve now runs through bin 2 of the batch
    assert lus[2]._fb is None and lus[2]._set_fb is not None
    assert _rel(lus[2].solve(b), ref.solve(b)) < 1e-12
    assert _rel(lus[2].solve(b, trans="T"), ref.solve(b, trans="T")) < 1e-12
    assert _rel(oadj.apply_monodromy_adjoint(Z["mono_v"], lus), Z["mono_MTv"]) < 1e-12
    orbit, info = oorb.solve_orbit_one_species(lus, list(SPC.emis), tol=1e-12)
    assert _rel(np.stack(orbit), Z["orbit"]) < 1e-9
    assert set(info) == {"gmres_iters", "residual", "periodicity", "neg_frac"}
    adj, ainfo = oadj.solve_orbit_adjoint_one_species(lus, list(Z["adj_R"]), tol=1e-12)
    assert _rel(np.stack(adj), Z["adjoint"]) < 1e-9
    g = oadj.gradient_per_emission_bin(adj, list(Z["adj_R"]))
    assert len(g) == 8 and g[0].shape == (MET[0].N,)
    # compute_s against the oracle sweep
    lus_cpu = [oorbit.factor_one_bin(Lt) for Lt in L]
    assert _rel(oorb.compute_s(lus, list(SPC.emis)), oorbit.compute_s(lus_cpu, list(SPC.emis))) < 1e-12


def test_all_species_with_coupling():
    """Three species, species 1 fed by species 0 through a diagonal K block
    (the SO2 -> pSO4 form), one zero-source species; wave 0 solves two species
    in one device batch."""
    from orbit_b200 import orbit as oorb
    N = MET[0].N
    L0 = _L_list(1.0)
    L1 = _L_list(2.0)
    L2 = _L_list(0.5)
    L_species = [[L0[t], L1[t], L2[t]] for t in range(8)]
    rate = 3e-5 * np.ones(N)
    K = [{(1, 0): sp.diags(-rate).tocsc()} for _ in range(8)]
    emis = np.zeros((8, 3 * N))
    emis[:, 0:N] = SPC.emis
    emis[:, N:2 * N] = 0.3 * SPC.emis
    res = oorb.solve_orbit_all_species([list(x) for x in L_species], K, emis, N, tol=1e-12, verbose=False)
    # oracle: species 0, then species 1 with e - K c0[tau]
    lus0 = [oorbit.factor_one_bin(L0[t]) for t in range(8)]
    o0, _ = oorbit.solve_orbit_one_species(lus0, list(SPC.emis), tol=1e-12)
    lus1 = [oorbit.factor_one_bin(L1[t]) for t in range(8)]
    e1 = [0.3 * SPC.emis[t] - K[t][(1, 0)] @ o0[t] for t in range(8)]
    o1, _ = oorbit.solve_orbit_one_species(lus1, e1, tol=1e-12)
    assert _rel(np.stack(res["orbits"][0]), np.stack(o0)) < 1e-9
    assert _rel(np.stack(res["orbits"][1]), np.stack(o1)) < 1e-9
    assert not np.any(np.stack(res["orbits"][2]))
    assert res["gmres_iters"][2] == 0


def test_operator_fct_massbalance_dropins():
    from orbit_b200 import operator as oop, fct as ofc
    from orbit_b200.grid import griddata_like
    grids = [griddata_like(g) for g in MET]
    T = oop.assemble_transport_block(grids[0])
    ref = golden_io.csc(Z, "T0_")
    assert _rel(T.toarray(), ref.toarray()) < 1e-12
    mb = oop.mass_balance_diagnostics(grids)
    got = np.array([mb[str(k)] for k in Z["mb_keys"]])
    np.testing.assert_allclose(got, Z["mb_vals"], rtol=1e-9, atol=1e-12)
    assert oop.gate(mb) == (Z["mb_vals"][1] <= 0.05)
    d = ofc.compute_horizontal_fct_source(grids[0], None, Z["fct_c"], 10800.0)
    assert _rel(d, Z["fct_d0"]) < 1e-12


def test_fct_deferred_passes_match_oracle():
    import torch
    from orbit_b200 import api, device
    from orbit_b200.symbolic import Symbolic
    L = _L_list()
    lus = [oorbit.factor_one_bin(Lt) for Lt in L]
    ref, rinfos = oorbit.fct_deferred_solve(lus, list(SPC.emis), MET, passes=2, tol=1e-12)
    mets = [device.MetDevice(g) for g in MET]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(x, device="cuda") for x in SPC.sink_diag(MET)]
    fb = device.FactorBatch(Symbolic(MET[0].nz, MET[0].ny, MET[0].nx), 1, 64)
    fb.numeric(T, sinks)
    orb, infos = api.solve_with_fct(fb, mets, torch.as_tensor(SPC.emis, device="cuda")[None], passes=2,
                                    tol=1e-12)
    assert len(infos) == 3
    assert _rel(orb[0].cpu().numpy(), np.stack(ref)) < 1e-9


def test_shared_operator_many_rhs():
    """Marginal-style right-hand sides on one operator, and adjoint receptors,
    all in one batch over a single factor set, equal the one-at-a-time solves."""
    import torch
    from orbit_b200 import api, device
    from orbit_b200.symbolic import Symbolic
    mets = [device.MetDevice(g) for g in MET]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(x, device="cuda") for x in SPC.sink_diag(MET)]
    sym = Symbolic(MET[0].nz, MET[0].ny, MET[0].nx)
    rng = np.random.default_rng(9)
    E = np.stack([SPC.emis * (1.0 + 0.1 * rng.standard_normal(SPC.emis.shape)) for _ in range(5)])
    Et = torch.as_tensor(E, device="cuda")
    orb, info = api.solve_shared_operator(sym, T, sinks, Et, precision=64, tol=1e-12)
    lus = [oorbit.factor_one_bin(Lt) for Lt in _L_list()]
    for q in range(5):
        ref, _ = oorbit.solve_orbit_one_species(lus, list(E[q]), tol=1e-12)
        assert _rel(orb[q].cpu().numpy(), np.stack(ref)) < 1e-9
    R = torch.as_tensor(np.stack([Z["adj_R"], 2 * Z["adj_R"]]), device="cuda")
    adj, _ = api.solve_shared_operator(sym, T, sinks, R, adjoint=True, precision=32, tol=1e-10)
    assert _rel(adj[0].cpu().numpy(), Z["adjoint"]) < 1e-6
    assert _rel(adj[1].cpu().numpy(), 2 * Z["adjoint"]) < 1e-6
