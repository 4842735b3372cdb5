"""CUDA path against the oracle and the reference's golden vectors (B200).

Tolerances: assembly, FCT and FP64 chained solves agree with the FP64 oracle
to 1e-12 relative (they differ only by floating-point association); FP64
periodic orbits solved at tol 1e-12 agree with the reference's to 1e-9 (max
over cells of |c - c_ref| / max|c_ref|); the mixed-precision path (FP32
factors, FP64 refinement) must stay within 1e-6.
"""
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
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def dev():
    import torch
    from orbit_b200 import device
    mets = [device.MetDevice(g) for g in MET]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(d, device="cuda") for d in SPC.sink_diag(MET)]
    return device, mets, T, sinks


def test_assembly_matches_reference(dev):
    device, mets, T, _ = dev
    g = MET[0]
    for t in range(8):
        A = device.stencil_to_csr(T[t].cpu().numpy(), g.nz, g.ny, g.nx)
        ref = golden_io.csc(Z, f"T{t}_")
        assert _rel(A.toarray(), ref.toarray()) < 1e-12


def test_rowsums_and_mass_balance(dev):
    device, mets, T, _ = dev
    _, rs = device.assemble_transport(mets[0], with_rowsum=True)
    Tp = assembly.transport_block(MET[0], concentration_form=False)
    ref = np.asarray(Tp.sum(axis=1)).ravel()
    assert np.abs(rs.cpu().numpy() - ref).max() <= 1e-12 * np.abs(Tp).max()
    mb = device.mass_balance(mets, T)
    got = np.array([mb[str(k)] for k in Z["mb_keys"]])
    np.testing.assert_allclose(got, Z["mb_vals"], rtol=1e-9, atol=1e-12)
    # identical gate decision at the reference's tolerance (cli.py:161, 1604-1615)
    assert (mb["interior_p90"] > 0.05) == (Z["mb_vals"][1] > 0.05)


def test_fct_source_matches_reference(dev):
    import torch
    device, mets, _, _ = dev
    c = torch.as_tensor(Z["fct_c"], device="cuda")
    for t in range(2):
        d = device.fct_source(mets[t], c).cpu().numpy()
        assert _rel(d, Z[f"fct_d{t}"]) < 1e-12
        du = device.fct_source(mets[t], c, limited=False).cpu().numpy()
        assert _rel(du, Z[f"fct_d{t}_unlim"]) < 1e-12
    # several vectors at once (one launch)
    cc = torch.stack([c, 2.0 * c, c.flip(0)])
    dd = device.fct_source(mets[0], cc).cpu().numpy()
    for q, cv in enumerate(cc.cpu().numpy()):
        assert _rel(dd[q], ofct.fct_source(MET[0], cv, 10800.0)) < 1e-12


def test_fct_linear_operator_matches_reference(dev):
    """Frozen-gain L_AD (fct.py:495-572) against the reference's CSC (golden),
    the oracle for other baselines, and L_AD c = -d_AD(c) by construction."""
    import torch
    device, mets, _, _ = dev
    g = MET[0]
    c = torch.as_tensor(Z["fct_c"], device="cuda")
    st = device.fct_linear_operator(mets[0], c).cpu().numpy()
    L = device.stencil_to_csr(st, g.nz, g.ny, g.nx)
    ref = golden_io.csc(Z, "fct_L0_")
    assert abs(L - ref).max() <= 1e-12 * abs(ref).max()
    assert _rel(L @ Z["fct_c"], -Z["fct_d0"]) < 1e-11
    cc = torch.stack([c, 3.0 * c.flip(0)])
    sts = device.fct_linear_operator(mets[1], cc).cpu().numpy()
    for q, cv in enumerate(cc.cpu().numpy()):
        want = ofct.fct_linear_operator(MET[1], cv, 10800.0)
        got = device.stencil_to_csr(sts[q], g.nz, g.ny, g.nx)
        assert abs(got - want).max() <= 1e-12 * abs(want).max()
    assert np.all(sts[:, 5:] == 0.0)  # horizontal only: vertical entries stay zero


def _batch(dev, precision=64, n=1):
    from orbit_b200.symbolic import Symbolic
    device, mets, T, sinks = dev
    g = MET[0]
    sym = Symbolic(g.nz, g.ny, g.nx, leaf_cells=8)
    fb = device.FactorBatch(sym, n, precision)
    fb.numeric(T * n, sinks * n)
    return fb


def test_monodromy_chain_matches_reference(dev):
    import torch
    fb = _batch(dev)
    v = torch.as_tensor(Z["mono_v"], device="cuda")[None]
    Mv = fb.chain(v).cpu().numpy()[0]
    assert _rel(Mv, Z["mono_Mv"]) < 1e-12
    MTv = fb.chain(v, trans=True).cpu().numpy()[0]
    assert _rel(MTv, Z["mono_MTv"]) < 1e-12


def test_single_bin_solves(dev):
    import torch
    device, mets, T, sinks = dev
    fb = _batch(dev)
    d = SPC.sink_diag(MET)
    rng = np.random.default_rng(5)
    b = rng.standard_normal(MET[0].N)
    for t in (0, 3, 7):
        A = sp.eye(MET[0].N) + 10800.0 * assembly.species_operator(assembly.transport_block(MET[t]), d[t])
        lu = sp.linalg.splu(A.tocsc())
        x = fb.chain(torch.as_tensor(b, device="cuda")[None], tau0=t, tau1=t + 1).cpu().numpy()[0]
        assert _rel(x, lu.solve(b)) < 1e-12
        xt = fb.chain(torch.as_tensor(b, device="cuda")[None], trans=True, tau0=t, tau1=t + 1).cpu().numpy()[0]
        assert _rel(xt, lu.solve(b, trans="T")) < 1e-12


def test_orbit_fp64_matches_reference(dev):
    import torch
    fb = _batch(dev)
    e = torch.as_tensor(SPC.emis, device="cuda")[None]
    orb, info = fb.solve(e, tol=1e-12)
    assert _rel(orb.cpu().numpy()[0], Z["orbit"]) < 1e-9
    assert info[0, 4] == 1.0 and info[0, 1] < 1e-11
    assert abs(info[0, 2] - Z["orbit_info"][2]) < 1e-9


def test_adjoint_fp64_matches_reference(dev):
    import torch
    fb = _batch(dev)
    R = torch.as_tensor(Z["adj_R"], device="cuda")[None]
    adj, info = fb.solve_adjoint(R, tol=1e-12)
    assert _rel(adj.cpu().numpy()[0], Z["adjoint"]) < 1e-9
    assert info[0, 2] < 1e-8


def test_mixed_precision_within_1e6(dev):
    import torch
    fb = _batch(dev, precision=32)
    e = torch.as_tensor(SPC.emis, device="cuda")[None]
    orb, info = fb.solve(e, tol=1e-8)
    assert _rel(orb.cpu().numpy()[0], Z["orbit"]) < 1e-6
    R = torch.as_tensor(Z["adj_R"], device="cuda")[None]
    adj, ainfo = fb.solve_adjoint(R, tol=1e-8)
    assert _rel(adj.cpu().numpy()[0], Z["adjoint"]) < 1e-6
    # the block-cyclic refinement's residual is the adjoint residual, and the
    # periodic closure holds: lam_8 = lam_0
    assert ainfo[0, 4] == 1.0 and ainfo[0, 1] <= 1e-8
    a = adj.cpu().numpy()[0]
    assert np.array_equal(a[0], a[8])
    # warm-started from the solution, the refinement stops at its first check
    adj2, ainfo2 = fb.solve_adjoint(R, lam_warm=adj[:, 0].contiguous(), tol=1e-8)
    assert _rel(adj2.cpu().numpy()[0], Z["adjoint"]) < 1e-6
    assert ainfo2[0, 6] <= 1


def test_batched_equals_alone(dev):
    """Orbits solved in one batch equal the same orbits solved alone."""
    import torch
    device, mets, T, sinks = dev
    fb3 = _batch(dev, n=3)
    e1 = torch.as_tensor(SPC.emis, device="cuda")
    e = torch.stack([e1, 3.0 * e1, e1.roll(7, dims=1)])
    orb3, _ = fb3.solve(e, tol=1e-12)
    fb1 = _batch(dev, n=1)
    for q in range(3):
        o1, _ = fb1.solve(e[q:q + 1], tol=1e-12)
        assert _rel(orb3[q].cpu().numpy(), o1[0].cpu().numpy()) < 1e-10


def test_config0_against_oracle():
    """Config-0 workload (24x20x15, one species): FP64 device orbit vs the
    SuperLU oracle at tol 1e-12; the device solve runs at the config's 1e-10."""
    import torch
    from orbit_b200 import device, synthetic
    from orbit_b200.symbolic import Symbolic
    wl = synthetic.config_workload(0)
    met = wl.met[0]
    sp0 = wl.species[0]
    d = sp0.sink_diag(met)
    lus = [oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(g), d[t]))
           for t, g in enumerate(met)]
    ref, rinfo = oorbit.solve_orbit_one_species(lus, list(sp0.emis), tol=1e-12)
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(x, device="cuda") for x in d]
    sym = Symbolic(wl.nz, wl.ny, wl.nx)
    fb = device.FactorBatch(sym, 1, 64)
    fb.numeric(T, sinks)
    orb, info = fb.solve(torch.as_tensor(sp0.emis, device="cuda")[None], tol=wl.tol)
    assert _rel(orb.cpu().numpy()[0], np.stack(ref)) < 1e-8
    fb32 = device.FactorBatch(sym, 1, 32)
    fb32.numeric(T, sinks)
    orb32, _ = fb32.solve(torch.as_tensor(sp0.emis, device="cuda")[None], tol=1e-8)
    assert _rel(orb32.cpu().numpy()[0], np.stack(ref)) < 1e-6


def test_pressure_form_grid_matches_reference():
    """A grid with concentration_state False through the drop-in modules: the
    block as assembled, unit state weights in the FCT source, L_AD and the
    mass-balance rows, against the reference's own outputs (golden)."""
    from orbit_b200 import fct as dfct, operator as dop
    from orbit_b200.grid import griddata_like
    zp, m = golden_io.load_pressure_form()
    g = griddata_like(m)
    assert g.concentration_state is False
    T = dop.assemble_transport_block(g)
    assert _rel(T.toarray(), golden_io.csc(zp, "pf_T_").toarray()) < 1e-12
    c = zp["pf_c"]
    assert _rel(dfct.compute_horizontal_fct_source(g, None, c, 10800.0), zp["pf_fct_d"]) < 1e-12
    assert _rel(dfct.compute_horizontal_fct_source(g, None, c, 10800.0, limited=False), zp["pf_fct_d_unlim"]) < 1e-12
    L = dfct.assemble_fct_linear_operator(g, None, c, 10800.0)
    assert _rel(L.toarray(), golden_io.csc(zp, "pf_fct_L_").toarray()) < 1e-12
    mb = dop.mass_balance_diagnostics([g])
    got = np.array([mb[str(k)] for k in zp["pf_mb_keys"]])
    np.testing.assert_allclose(got, zp["pf_mb_vals"], rtol=1e-9, atol=1e-12)
