"""Species operators: sink diagonals and source couplings of
assemble_species_operators (orbit/core/operator.py:371-595) against the
reference's own outputs (tests/golden/species_ops.npz, written by
tests/golden/make_golden.py --species).

The CPU oracle (oracle/species.py) must reproduce the reference to 1e-14
relative on both grids ('full': every optional field, the photolytic sink on,
the VBS aging cascade; 'min': only the required fields, the reference's
fallbacks) and both partitionings.  The device drop-in
(orbit_b200.operator.assemble_species_operators, kernel K1b) is checked the
same way on a B200, including the transport block and one full L_s.
"""
import os

import numpy as np
import pytest

import golden_io
from oracle import species as ospecies

HERE = os.path.dirname(os.path.abspath(__file__))
Z = dict(np.load(os.path.join(HERE, "golden", "species_ops.npz")))
A_PHOTO = 4.0e-4


def _grid(tag):
    from orbit_b200.grid import griddata_like
    m = golden_io.met_bin(Z, "sp_")
    g = griddata_like(m)
    keys = [k[len("full_"):] for k in Z if k.startswith("full_") and not k.startswith("full_marginal")
            and not k.startswith("full_equilibrium")]
    if tag == "full":
        for k in keys:
            setattr(g, k, Z[f"full_{k}"])
    else:
        for k in ("particle_dry_dep", "NH3_dry_dep", "SO2_dry_dep", "NOx_dry_dep", "particle_wet_dep",
                  "other_gas_wet_dep", "SO2_wet_dep", "NHPartitioning"):
            setattr(g, k, Z[f"full_{k}"])
    return g


def _rates(tag):
    if tag == "full":
        return {k[len("rate_"):]: Z[k] for k in Z if k.startswith("rate_")}
    return {"so2_ox_rate": Z["so2_override"]}


CASES = [(t, p) for t in ("full", "min") for p in ("marginal", "equilibrium")]


def _close(a, b, rtol):
    return np.abs(np.asarray(a) - np.asarray(b)).max() <= rtol * max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("tag,part", CASES)
def test_oracle_species_diagonals_match_reference(tag, part):
    g = _grid(tag)
    r = _rates(tag)
    d, K, D, Kage = ospecies.diagonals(g, part, a_photo=A_PHOTO, so2_ox=r.get("so2_ox_rate"),
                                       nox_ox=r.get("nox_to_no3_rate"), o3_loss=r.get("o3_loss_rate"),
                                       co_loss=r.get("co_loss_rate"))
    key = f"{tag}_{part}"
    assert _close(d, Z[f"{key}_d"], 1e-14)
    assert _close(D, Z[f"{key}_D"], 1e-14)
    keys = [tuple(k) for k in Z[f"{key}_Kkeys"]]
    assert sorted(K.keys()) == keys
    for q, k in enumerate(keys):
        assert _close(K[k], Z[f"{key}_Kdiag"][q], 1e-14)
    assert sorted(Kage.keys()) == list(Z[f"{key}_Kagekeys"])
    for q, k in enumerate(sorted(Kage.keys())):
        assert _close(Kage[k], Z[f"{key}_Kage"][q], 1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("tag,part", CASES)
def test_device_species_operators_match_reference(tag, part, monkeypatch):
    from orbit_b200 import operator as dop
    monkeypatch.setenv("ORBIT_VBS_A_PHOTO", str(A_PHOTO))
    g = _grid(tag)
    r = _rates(tag)
    L, K, T, d, D, Kage = dop.assemble_species_operators(g, None, verbose=False, return_D_per_species=True,
                                                         partitioning=part, **r)
    key = f"{tag}_{part}"
    assert _close(d, Z[f"{key}_d"], 1e-14)
    assert _close(np.stack([x.diagonal() for x in D]), Z[f"{key}_D"], 1e-14)
    keys = [tuple(k) for k in Z[f"{key}_Kkeys"]]
    assert sorted(K.keys()) == keys
    for q, k in enumerate(keys):
        assert _close(K[k].diagonal(), Z[f"{key}_Kdiag"][q], 1e-14)
    assert sorted(Kage.keys()) == list(Z[f"{key}_Kagekeys"])
    for q, k in enumerate(sorted(Kage.keys())):
        assert _close(Kage[k].diagonal(), Z[f"{key}_Kage"][q], 1e-14)
    Tref = golden_io.csc(Z, f"{key}_T_")
    assert _close(T.toarray(), Tref.toarray(), 1e-12)
    assert _close(L[1].toarray(), golden_io.csc(Z, f"{key}_L1_").toarray(), 1e-12)


NOX = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nox_rate.npz")))


def _nox_grid(tag):
    from types import SimpleNamespace
    g = SimpleNamespace(nz=4, ny=5, nx=6)
    for k in ("Temperature", "Pressure", "archive_OH", "archive_NO", "archive_NO2", "archive_NO3rad", "pS", "pNH",
              "pNO", "dust_fine", "sea_salt_fine"):
        setattr(g, k, NOX[f"nx_{k}"])
    if tag == "lean":
        for k in ("archive_NO", "archive_NO3rad", "pNO", "dust_fine"):
            setattr(g, k, np.array([]))
    return g


@pytest.mark.parametrize("tag", ["full", "lean"])
def test_oracle_nox_rate_matches_reference(tag):
    """build_nox_to_no3_rate (nox_to_no3_rate.py:94-155): day + night and day only."""
    from oracle import species as osp
    g = _nox_grid(tag)
    ref = NOX[f"nx_rate_{tag}"]
    assert np.abs(osp.nox_to_no3_rate(g) - ref).max() <= 1e-12 * np.abs(ref).max()
    ref_d = NOX[f"nx_rate_{tag}_day"]
    assert np.abs(osp.nox_to_no3_rate(g, disable_night=True) - ref_d).max() <= 1e-12 * np.abs(ref_d).max()


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["full", "lean"])
def test_device_nox_rate_matches_reference(tag):
    """K1b NOx -> TotalNO3 rate through the build_nox_to_no3_rate drop-in."""
    from orbit_b200 import operator as dop
    g = _nox_grid(tag)
    for night, key in ((False, f"nx_rate_{tag}"), (True, f"nx_rate_{tag}_day")):
        got = dop.build_nox_to_no3_rate(g, disable_night=night)
        ref = NOX[key]
        assert got.shape == ref.shape
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    g.archive_OH = np.array([])
    assert dop.build_nox_to_no3_rate(g) is None
