"""Orbit NPZ files in the reference's layout (orbit/cli.py:1297-1408): the keys
_save_checkpoint writes, the state _load_checkpoint restores, and the
adjoint's FCT baseline read (orbit/modes/adjoint.py:548-565)."""
import numpy as np

from orbit_b200 import io


def _result(rng, N=30):
    orbits = {3: [rng.random(N) for _ in range(9)], 0: [rng.random(N) for _ in range(9)],
              5: [rng.random(N) for _ in range(9)]}
    return {"orbits": orbits, "gmres_iters": np.array([4, 0, 0, 7, 0, 3]),
            "gmres_resid": rng.random(6), "periodicity": rng.random(6)}


def test_round_trip_and_keys(tmp_path):
    rng = np.random.default_rng(1)
    res = _result(rng)
    p = io.save_orbit_npz(str(tmp_path / "orbit_M01_iter03.npz"), res, month=1, it=3, converged=False,
                          closure_mode="anderson", closure_alpha=0.5, closure_tol=1e-3, grid_shape=(2, 3, 5))
    with np.load(p) as d:
        assert {"month", "iter", "converged", "closure_mode", "closure_alpha", "closure_tol", "grid_shape",
                "c_orbit", "orbit_species_order", "gmres_iters", "gmres_resid", "periodicity"} <= set(d.files)
        assert d["c_orbit"].shape == (3, 9, 30)
        assert list(d["orbit_species_order"]) == [0, 3, 5]
    st = io.load_orbit_npz(p)
    assert st["iter"] == 3 and st["converged"] is False
    for s, o in res["orbits"].items():
        assert all(np.array_equal(a, b) for a, b in zip(st["orbits"][s], o))
    np.testing.assert_array_equal(st["gmres_iters"], res["gmres_iters"])
