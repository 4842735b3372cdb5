"""Periodic-longitude grids and the lateral boundary loss on the device,
against the reference's outputs (tests/golden/periodic.npz) and the oracle.

* K1 with the wrap face (convdiff.py:150-202), split and non-split (meander)
  modes, and through the assemble_transport_block drop-in: 1e-12;
* the lateral boundary loss (return_boundary_fluxes, operator.py:25-178,
  344-347) of periodic and regional grids: 1e-12;
* stencil products with the wrap couplings, forward and transposed: 1e-13;
* bin solves and the chained monodromy through the ring dissection: 1e-12
  against SuperLU; the FP64 periodic orbit at tol 1e-12 against the
  reference's: 1e-9; the mixed-precision orbit: 1e-6; the adjoint orbit
  against the oracle's: 1e-9;
* the FCT source of a periodic grid (the reference's FCT has no wrap face): 1e-12.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import golden_io
from oracle import assembly, orbit as oorbit
from orbit_b200 import synthetic

pytestmark = pytest.mark.gpu

Z = golden_io.load_periodic()


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_wrap_face_assembly_matches_reference():
    from orbit_b200 import device, operator as dop
    from orbit_b200.grid import griddata_like
    for tag in ("ps_", "pn_"):
        m = golden_io.met_bin(Z, tag)
        md = device.MetDevice(m)
        st = device.assemble_transport(md).cpu().numpy()
        T = device.stencil_to_csr(st, m.nz, m.ny, m.nx, periodic=True)
        ref = golden_io.csc(Z, f"{tag}T_")
        assert abs(T - ref).max() <= 1e-12 * abs(ref).max()
        Td, loss = dop.assemble_transport_block(griddata_like(m), return_boundary_fluxes=True)
        assert abs(Td - ref).max() <= 1e-12 * abs(ref).max()
        assert np.abs(loss - Z[f"{tag}loss"]).max() <= 1e-12 * max(np.abs(Z[f"{tag}loss"]).max(), 1e-300)


def test_boundary_loss_matches_reference():
    from orbit_b200 import device
    for tag in ("ps_", "pn_", "rs_", "rn_"):
        m = golden_io.met_bin(Z, tag)
        loss = device.boundary_loss(device.MetDevice(m)).cpu().numpy()
        ref = Z[f"{tag}loss"]
        assert np.abs(loss - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-300)


def test_wrapped_stencil_products():
    import torch
    from orbit_b200 import device
    m = golden_io.met_bin(Z, "ps_")
    st = device.assemble_transport(device.MetDevice(m))
    T = device.stencil_to_csr(st.cpu().numpy(), m.nz, m.ny, m.nx, periodic=True)
    x = np.random.default_rng(3).standard_normal(m.N)
    xt = torch.as_tensor(x, device="cuda")
    y = device.stencil_apply(m.nz, m.ny, m.nx, st, xt, periodic=True).cpu().numpy()
    assert _rel(y, T @ x) < 1e-13
    yt = device.stencil_apply(m.nz, m.ny, m.nx, st, xt, trans=True, periodic=True).cpu().numpy()
    assert _rel(yt, T.T @ x) < 1e-13


@pytest.fixture(scope="module")
def orbit_case():
    import torch
    from orbit_b200 import device
    met = [golden_io.met_bin(Z, f"om{t}_") for t in range(8)]
    spc = synthetic.SpeciesFields(vd=Z["o_vd"], wet=Z["o_wet"], loss=Z["o_loss"], emis=Z["o_emis"])
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(md) for md in mets]
    sinks = [torch.as_tensor(d, device="cuda") for d in spc.sink_diag(met)]
    return met, spc, T, sinks


def _batch(orbit_case, precision):
    from orbit_b200 import device
    from orbit_b200.symbolic import Symbolic
    met, spc, T, sinks = orbit_case
    g = met[0]
    sym = Symbolic(g.nz, g.ny, g.nx, leaf_cells=8, periodic=True)
    fb = device.FactorBatch(sym, 1, precision)
    fb.numeric(T, sinks)
    return fb


def test_periodic_bin_solves_and_monodromy(orbit_case):
    import torch
    met, spc, T, sinks = orbit_case
    fb = _batch(orbit_case, 64)
    d = spc.sink_diag(met)
    g = met[0]
    b = np.random.default_rng(4).standard_normal(g.N)
    lus = []
    for t in range(8):
        A = (sp.eye(g.N) + 10800.0 * assembly.species_operator(assembly.transport_block(met[t]), d[t])).tocsc()
        lu = sp.linalg.splu(A)
        lus.append(lu)
        bt = torch.as_tensor(b, device="cuda")[None]
        assert _rel(fb.chain(bt, tau0=t, tau1=t + 1).cpu().numpy()[0], lu.solve(b)) < 1e-12
        assert _rel(fb.chain(bt, trans=True, tau0=t, tau1=t + 1).cpu().numpy()[0], lu.solve(b, trans="T")) < 1e-12
    v = b.copy()
    for t in range(8):
        v = lus[t].solve(v)
    assert _rel(fb.chain(torch.as_tensor(b, device="cuda")[None]).cpu().numpy()[0], v) < 1e-12


def test_periodic_orbit_matches_reference(orbit_case):
    import torch
    met, spc, T, sinks = orbit_case
    e = torch.as_tensor(spc.emis, device="cuda")[None]
    orb, info = _batch(orbit_case, 64).solve(e, tol=1e-12)
    assert _rel(orb.cpu().numpy()[0], Z["o_orbit"]) < 1e-9
    orb32, _ = _batch(orbit_case, 32).solve(e, tol=1e-8)
    assert _rel(orb32.cpu().numpy()[0], Z["o_orbit"]) < 1e-6


def test_periodic_adjoint_matches_oracle(orbit_case):
    import torch
    met, spc, T, sinks = orbit_case
    d = spc.sink_diag(met)
    lus = [oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(g), d[t]))
           for t, g in enumerate(met)]
    R = np.abs(np.random.default_rng(6).standard_normal((8, met[0].N)))
    ref, _ = oorbit.solve_orbit_adjoint_one_species(lus, list(R), tol=1e-12)
    adj, _ = _batch(orbit_case, 64).solve_adjoint(torch.as_tensor(R, device="cuda")[None], tol=1e-12)
    assert _rel(adj.cpu().numpy()[0], np.stack(ref)) < 1e-9


def test_fct_source_on_periodic_grid():
    import torch
    from orbit_b200 import device
    for tag in ("ps_", "pn_"):
        m = golden_io.met_bin(Z, tag)
        c = torch.as_tensor(Z[f"{tag}c"], device="cuda")
        d = device.fct_source(device.MetDevice(m), c).cpu().numpy()
        assert _rel(d, Z[f"{tag}fct_d"]) < 1e-12


def test_fct_ghost_field_matches_reference():
    """Lateral-inflow field (c_ghost_flat, fct.py:283-292, 381-400): limited
    and unlimited sources against the reference, the drop-in's signature, and
    several vectors with their own ghost fields in one launch against the oracle."""
    import torch
    from orbit_b200 import device, fct as dfct
    from oracle import fct as ofct
    from orbit_b200.grid import griddata_like
    for tag in ("rs_", "rn_"):
        m = golden_io.met_bin(Z, tag)
        md = device.MetDevice(m)
        c = torch.as_tensor(Z[f"{tag}c"], device="cuda")
        cg = torch.as_tensor(Z[f"{tag}cg"], device="cuda")
        assert _rel(device.fct_source(md, c, c_ghost=cg).cpu().numpy(), Z[f"{tag}fct_dg"]) < 1e-12
        assert _rel(device.fct_source(md, c, limited=False, c_ghost=cg).cpu().numpy(),
                    Z[f"{tag}fct_dg_unlim"]) < 1e-12
        got = dfct.compute_horizontal_fct_source(griddata_like(m), None, Z[f"{tag}c"], 10800.0,
                                                 c_ghost_flat=Z[f"{tag}cg"])
        assert _rel(got, Z[f"{tag}fct_dg"]) < 1e-12
        cc = torch.stack([c, 2.0 * c.flip(0)])
        gg = torch.stack([cg, 0.5 * cg])
        dd = device.fct_source(md, cc, c_ghost=gg).cpu().numpy()
        for q in range(2):
            ref = ofct.fct_source(m, cc[q].cpu().numpy(), 10800.0, c_ghost_flat=gg[q].cpu().numpy())
            assert _rel(dd[q], ref) < 1e-12


def test_periodic_orbit_through_the_dropin_modules():
    """The reference's call sequence on a periodic grid: umfpack_symbolic(L)
    recognises the wrap couplings of the CSC operator, _factor_one_bin gives
    the device LU objects, solve_orbit_one_species the orbit (reference golden
    at 1e-9); the LU objects' transposed solves match SuperLU's."""
    from orbit_b200 import orbit as dorb
    from orbit_b200.solve import umfpack_symbolic
    met = [golden_io.met_bin(Z, f"om{t}_") for t in range(8)]
    spc = synthetic.SpeciesFields(vd=Z["o_vd"], wet=Z["o_wet"], loss=Z["o_loss"], emis=Z["o_emis"])
    d = spc.sink_diag(met)
    L = [assembly.species_operator(assembly.transport_block(g), d[t]).tocsc() for t, g in enumerate(met)]
    sym = umfpack_symbolic(L[0], verbose=False)
    assert sym.sym.periodic
    N = met[0].N
    I_N = sp.identity(N, format="csc")
    lus = [dorb._factor_one_bin(L[t], I_N, sym, None) for t in range(8)]
    orb, info = dorb.solve_orbit_one_species(lus, [spc.emis[t] for t in range(8)], tol=1e-12)
    assert _rel(np.stack(orb), Z["o_orbit"]) < 1e-9
    b = np.random.default_rng(9).standard_normal(N)
    A = (I_N + 10800.0 * L[3]).tocsc()
    ref = sp.linalg.splu(A)
    assert _rel(lus[3].solve(b, trans="T"), ref.solve(b, trans="T")) < 1e-12
