"""The closure loop around the orbit solve: the ISORROPIA 7-D LUT query
(orbit/core/isorropia_lut.py:116-147) and the Anderson step
(orbit/core/closure_iteration.py:568-694), against the reference's own
outputs (tests/golden/closure.npz, tests/golden/make_golden.py --closure):
a synthetic table in the reference's file layout queried inside, on grid
nodes and outside its axes (extrapolation), and Anderson sequences with and
without the safeguard on a linear fixed-point map.  The CPU oracle is pinned
first; the device versions (kernel orbit_lut_query, orbit_vec_dots /
orbit_vec_combine) follow on a B200.
"""
import os

import numpy as np
import pytest

from oracle import closure as ocl

HERE = os.path.dirname(os.path.abspath(__file__))
Z = dict(np.load(os.path.join(HERE, "golden", "closure.npz")))
AXES = ("so4_axis", "nh_axis", "no3_axis", "ca_axis", "na_axis", "t_axis", "rh_axis")
FIELDS = ("f_nh4", "f_no3", "aerosol_water", "ph")


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.nanmax(np.abs(a - b)) / max(np.nanmax(np.abs(b)), 1e-300))


def _sequence(acc, tag, guarded):
    A, b = Z["and_A"], Z["and_b"]
    x = np.zeros(len(b))
    xs, oks = [x.copy()], []
    for _ in range(10):
        if guarded:
            x, ok = acc.apply_with_safeguard(x, A @ x + b)
            oks.append(ok)
        else:
            x = acc.update(x, A @ x + b)
        xs.append(np.asarray(x).copy())
    return np.stack(xs), oks


KW = {"m3": dict(m=3, beta=1.0), "m2d": dict(m=2, beta=0.6, safeguard_factor=1.05)}


def test_oracle_lut_query_matches_reference():
    axes = [Z[f"lut_{a}"] for a in AXES]
    out = ocl.lut_query(axes, [Z[f"lut_{f}"] for f in FIELDS], Z["lut_pts"])
    assert _rel(np.stack(out), Z["lut_out"]) < 1e-12
    out2 = ocl.lut_query(axes, [Z["lut_f_nh4"], Z["lut_f_no3"], None, None], Z["lut_pts"])
    assert _rel(np.stack(out2)[:2], Z["lut_out_two_fields"][:2]) < 1e-12
    assert np.all(np.isnan(np.stack(out2)[2:])) and np.all(np.isnan(Z["lut_out_two_fields"][2:]))


@pytest.mark.parametrize("tag", ["m3", "m2d"])
def test_oracle_anderson_matches_reference(tag):
    xs, oks = _sequence(ocl.Anderson(**KW[tag]), tag, True)
    assert _rel(xs, Z[f"and_{tag}_x"]) < 1e-10
    assert oks == list(Z[f"and_{tag}_ok"])
    kw = {k: v for k, v in KW[tag].items() if k != "safeguard_factor"}
    xs, _ = _sequence(ocl.Anderson(**kw), tag, False)
    assert _rel(xs, Z[f"and_{tag}_x_unguarded"]) < 1e-10


@pytest.mark.gpu
def test_device_lut_query_matches_reference(tmp_path):
    from orbit_b200.isorropia import IsorropiaLUT
    path = tmp_path / "lut.npz"
    np.savez(path, **{a: Z[f"lut_{a}"] for a in AXES}, **{f: Z[f"lut_{f}"] for f in FIELDS})
    pts = Z["lut_pts"]
    lut = IsorropiaLUT(path, fields=FIELDS)
    out = lut.query(*[pts[:, d] for d in range(7)])
    assert _rel(np.stack(out), Z["lut_out"]) < 1e-12
    lut2 = IsorropiaLUT(path)
    out2 = np.stack(lut2.query(*[pts[:, d] for d in range(7)]))
    assert _rel(out2[:2], Z["lut_out_two_fields"][:2]) < 1e-12
    assert np.all(np.isnan(out2[2:]))
    lut2.release()
    assert not lut2.loaded
    assert _rel(np.stack(lut2.query(*[pts[:, d] for d in range(7)]))[:2], out2[:2]) == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["m3", "m2d"])
def test_device_anderson_matches_reference(tag):
    from orbit_b200.closure import AndersonAccelerator
    xs, oks = _sequence(AndersonAccelerator(**KW[tag]), tag, True)
    assert _rel(xs, Z[f"and_{tag}_x"]) < 1e-10
    assert oks == list(Z[f"and_{tag}_ok"])
    kw = {k: v for k, v in KW[tag].items() if k != "safeguard_factor"}
    xs, _ = _sequence(AndersonAccelerator(**kw), tag, False)
    assert _rel(xs, Z[f"and_{tag}_x_unguarded"]) < 1e-10
