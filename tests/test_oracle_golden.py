"""The CPU oracle against golden vectors produced by the reference itself."""
import numpy as np
import scipy.sparse as sp

import golden_io
from oracle import assembly, fct, orbit as oorbit

Z = golden_io.load()
MET = golden_io.met_list(Z)
SPC = golden_io.species(Z)


def _close(A, B, rtol=1e-12):
    d = abs(A - B)
    scale = abs(B).max()
    return d.max() <= rtol * scale


def test_patankar_known_answers():
    np.testing.assert_allclose(assembly.patankar_A(Z["pe"]), Z["patankar"], rtol=1e-14, atol=0)
    assert abs(assembly.patankar_A(np.array([1.0]))[0] - 1.0 / np.expm1(1.0)) < 1e-15


def test_blocks_match_reference():
    g = MET[0]
    assert _close(assembly.horizontal_convdiff(g), golden_io.csc(Z, "T0_hcd_"))
    assert _close(assembly.vertical_advection(g), golden_io.csc(Z, "T0_vadv_"))
    assert _close(assembly.vertical_diffusion(g), golden_io.csc(Z, "T0_vdiff_"))
    assert _close(assembly.cmfmc_transport(g), golden_io.csc(Z, "T0_conv_"))


def test_nonsplit_horizontal_block():
    g = golden_io.met_bin(Z, "ns_")
    assert _close(assembly.horizontal_convdiff(g), golden_io.csc(Z, "Tns_hcd_"))


def test_transport_block_all_bins():
    for t, g in enumerate(MET):
        assert _close(assembly.transport_block(g), golden_io.csc(Z, f"T{t}_"))


def test_deposition_diagonal():
    d = SPC.sink_diag(MET)
    for t in range(8):
        np.testing.assert_allclose(d[t], Z[f"D{t}"] + SPC.loss[t].reshape(-1), rtol=1e-14, atol=0)


def test_mass_balance():
    mb = assembly.mass_balance_diagnostics(MET)
    got = np.array([mb[str(k)] for k in Z["mb_keys"]])
    np.testing.assert_allclose(got, Z["mb_vals"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(mb["layer_p90"], Z["mb_layer_p90"], rtol=1e-9, atol=1e-12)


def test_fct_source():
    c = Z["fct_c"]
    for t in range(2):
        np.testing.assert_allclose(fct.fct_source(MET[t], c, 10800.0), Z[f"fct_d{t}"],
                                   rtol=1e-12, atol=1e-12 * np.abs(Z[f"fct_d{t}"]).max())
        np.testing.assert_allclose(fct.fct_source(MET[t], c, 10800.0, limited=False),
                                   Z[f"fct_d{t}_unlim"], rtol=1e-12,
                                   atol=1e-12 * np.abs(Z[f"fct_d{t}_unlim"]).max())
    g = golden_io.met_bin(Z, "ns_")
    np.testing.assert_allclose(fct.fct_source(g, c, 10800.0), Z["fct_dns"], rtol=1e-12,
                               atol=1e-12 * np.abs(Z["fct_dns"]).max())
    assert _close(fct.fct_linear_operator(MET[0], c, 10800.0), golden_io.csc(Z, "fct_L0_"))


def _lus():
    d = SPC.sink_diag(MET)
    return [oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(g), d[t]))
            for t, g in enumerate(MET)]


def test_monodromy_and_adjoint_chain():
    lus = _lus()
    np.testing.assert_allclose(oorbit.apply_monodromy(Z["mono_v"], lus), Z["mono_Mv"], rtol=1e-12,
                               atol=1e-13 * np.abs(Z["mono_Mv"]).max())
    np.testing.assert_allclose(oorbit.apply_monodromy_adjoint(Z["mono_v"], lus), Z["mono_MTv"],
                               rtol=1e-12, atol=1e-13 * np.abs(Z["mono_MTv"]).max())


def test_orbit_solve():
    lus = _lus()
    orb, info = oorbit.solve_orbit_one_species(lus, list(SPC.emis), tol=1e-12)
    ref = Z["orbit"]
    err = np.abs(np.stack(orb) - ref).max() / np.abs(ref).max()
    assert err < 1e-10
    assert info["residual"] < 1e-11


def test_adjoint_solve():
    lus = _lus()
    adj, info = oorbit.solve_orbit_adjoint_one_species(lus, list(Z["adj_R"]), tol=1e-12)
    ref = Z["adjoint"]
    err = np.abs(np.stack(adj) - ref).max() / np.abs(ref).max()
    assert err < 1e-10
    assert info["periodicity"] < 1e-8


def test_pressure_form_grid():
    """concentration_state False: no similarity transform, unit state weights
    in the FCT source, L_AD and the mass-balance rows (operator.py:341,
    fct.py:451-456, operator.py:626)."""
    zp, g = golden_io.load_pressure_form()
    assert _close(assembly.transport_block(g), golden_io.csc(zp, "pf_T_"))
    c = zp["pf_c"]
    np.testing.assert_allclose(fct.fct_source(g, c, 10800.0), zp["pf_fct_d"], rtol=1e-12,
                               atol=1e-12 * np.abs(zp["pf_fct_d"]).max())
    np.testing.assert_allclose(fct.fct_source(g, c, 10800.0, limited=False), zp["pf_fct_d_unlim"],
                               rtol=1e-12, atol=1e-12 * np.abs(zp["pf_fct_d_unlim"]).max())
    assert _close(fct.fct_linear_operator(g, c, 10800.0), golden_io.csc(zp, "pf_fct_L_"))
    mb = assembly.mass_balance_diagnostics([g])
    got = np.array([mb[str(k)] for k in zp["pf_mb_keys"]])
    np.testing.assert_allclose(got, zp["pf_mb_vals"], rtol=1e-9, atol=1e-12)
