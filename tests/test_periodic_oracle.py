"""Periodic-longitude grids and the lateral boundary loss on the CPU: the
oracle against the reference's own outputs (tests/golden/periodic.npz, made
by tests/golden/make_golden.py --periodic), and the dissection of a
longitude ring replayed on the host.

* transport block with the wrap face (convdiff.py:150-202), split and
  non-split (meander) flux modes: 1e-12 relative;
* compute_lateral_boundary_loss (operator.py:25-178) of periodic and
  regional grids: 1e-12;
* the FCT source of a periodic grid (fct.py, no wrap face): 1e-12;
* a periodic orbit solved with SuperLU on the oracle's blocks (tol 1e-12)
  against the reference's: 1e-9.
"""
import numpy as np
import scipy.sparse as sp

import golden_io
from oracle import assembly, fct as ofct, orbit as oorbit
from orbit_b200 import synthetic

Z = golden_io.load_periodic()


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_wrap_face_block_matches_reference():
    for tag in ("ps_", "pn_"):
        m = golden_io.met_bin(Z, tag)
        assert m.periodic_lon
        T = assembly.transport_block(m)
        ref = golden_io.csc(Z, f"{tag}T_")
        assert abs(T - ref).max() <= 1e-12 * abs(ref).max()
        # the wrap couplings are there: column 0 <-> column nx-1
        nx = m.nx
        assert ref[0, nx - 1] != 0.0 and ref[nx - 1, 0] != 0.0


def test_lateral_boundary_loss_matches_reference():
    for tag in ("ps_", "pn_", "rs_", "rn_"):
        m = golden_io.met_bin(Z, tag)
        loss = assembly.lateral_boundary_loss(m)
        ref = Z[f"{tag}loss"]
        assert np.abs(loss - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-300)
        L3 = ref.reshape(m.nz, m.ny, m.nx)
        assert np.all(L3[:, 1:-1, 1:-1] == 0.0)
        if m.periodic_lon:  # no x-boundary loss on a periodic grid
            assert np.all(L3[:, 1:-1, :] == 0.0)


def test_fct_source_on_periodic_grid_matches_reference():
    for tag in ("ps_", "pn_"):
        m = golden_io.met_bin(Z, tag)
        d = ofct.fct_source(m, Z[f"{tag}c"], 10800.0)
        assert _rel(d, Z[f"{tag}fct_d"]) < 1e-12


def test_periodic_orbit_matches_reference():
    met = [golden_io.met_bin(Z, f"om{t}_") for t in range(8)]
    spc = synthetic.SpeciesFields(vd=Z["o_vd"], wet=Z["o_wet"], loss=Z["o_loss"], emis=Z["o_emis"])
    d = spc.sink_diag(met)
    lus = [oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(g), d[t]))
           for t, g in enumerate(met)]
    orb, _ = oorbit.solve_orbit_one_species(lus, list(spc.emis), tol=1e-12)
    assert _rel(np.stack(orb), Z["o_orbit"]) < 1e-9


def test_fct_ghost_field_matches_reference():
    """The lateral-inflow (ghost) field of compute_horizontal_fct_source
    (fct.py:283-292, 381-400, 476-487), limited and unlimited; without it the
    same grids give the edge-clamped source."""
    for tag in ("rs_", "rn_"):
        m = golden_io.met_bin(Z, tag)
        c, cg = Z[f"{tag}c"], Z[f"{tag}cg"]
        assert _rel(ofct.fct_source(m, c, 10800.0, c_ghost_flat=cg), Z[f"{tag}fct_dg"]) < 1e-12
        assert _rel(ofct.fct_source(m, c, 10800.0, limited=False, c_ghost_flat=cg), Z[f"{tag}fct_dg_unlim"]) < 1e-12
        assert _rel(ofct.fct_source(m, c, 10800.0), Z[f"{tag}fct_d"]) < 1e-12
        assert _rel(Z[f"{tag}fct_dg"], Z[f"{tag}fct_d"]) > 1e-6  # the ghost field matters here
