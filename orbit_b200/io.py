"""Orbit NPZ files in the reference's layout.

The forward driver writes the solved orbits of every species into an NPZ
(``_save_checkpoint``, orbit/cli.py:1297-1381) that later runs read back:
the resume path (``_load_checkpoint``, cli.py:1384-1408) and the adjoint's
FCT baseline (``c_orbit`` / ``orbit_species_order``, orbit/modes/adjoint.py:
548-565).  ``save_orbit_npz`` writes the same keys for a result of
``solve_orbit_all_species`` (device or host orbits), ``load_orbit_npz``
restores the state ``_load_checkpoint`` restores, and ``baseline_orbits``
hands a forward run's orbits to the device FCT operators
(``api.fct_operators``) the way the adjoint reads them.
"""
from __future__ import annotations

import os
from typing import Dict, Optional

import numpy as np


def _stack_orbits(orbits) -> (np.ndarray, np.ndarray):
    order = sorted(int(s) for s in orbits.keys())
    rows = []
    for s in order:
        o = orbits[s]
        if hasattr(o, "detach"):  # a (9, N) device tensor
            rows.append(o.detach().cpu().numpy())
        else:
            rows.append(np.stack([np.asarray(c, dtype=np.float64) for c in o], axis=0))
    return np.stack(rows, axis=0), np.array(order)


def save_orbit_npz(path: str, result: Dict, month: int, it: int = 0, converged: bool = True,
                   closure_mode: str = "none", closure_alpha: float = 1.0, closure_tol: float = 0.0,
                   grid_shape=None, extra: Optional[Dict[str, np.ndarray]] = None) -> str:
    """Write orbits and solver diagnostics with the reference's keys: month,
    iter, converged, closure_mode, closure_alpha, closure_tol, [grid_shape],
    c_orbit (n_species, 9, N), orbit_species_order, gmres_iters, gmres_resid,
    periodicity (cli.py:1309-1330), plus any ``extra`` arrays."""
    c_orbit, order = _stack_orbits(result["orbits"])
    save = {
        "month": np.array(month), "iter": np.array(it), "converged": np.array(converged, dtype=bool),
        "closure_mode": np.array(closure_mode), "closure_alpha": np.array(closure_alpha),
        "closure_tol": np.array(closure_tol),
        "c_orbit": c_orbit, "orbit_species_order": order,
        "gmres_iters": np.asarray(result["gmres_iters"]), "gmres_resid": np.asarray(result["gmres_resid"]),
        "periodicity": np.asarray(result["periodicity"]),
    }
    if grid_shape is not None:
        save["grid_shape"] = np.array(grid_shape)
    if extra:
        save.update({k: np.asarray(v) for k, v in extra.items()})
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    np.savez_compressed(path, **save)
    return path


def load_orbit_npz(path: str) -> Dict:
    """The state ``_load_checkpoint`` restores (cli.py:1384-1408): orbits per
    species as 9 arrays, gmres_iters, gmres_resid, periodicity, iter,
    converged, and the conv_* arrays."""
    with np.load(path, allow_pickle=False) as d:
        c_orbit = d["c_orbit"]
        order = d["orbit_species_order"]
        orbits = {int(s): [c_orbit[i, t].copy() for t in range(c_orbit.shape[1])]
                  for i, s in enumerate(order.tolist())}
        return {
            "orbits": orbits,
            "gmres_iters": d["gmres_iters"].copy(),
            "gmres_resid": d["gmres_resid"].copy(),
            "periodicity": d["periodicity"].copy(),
            "iter": int(d["iter"]),
            "converged": bool(d["converged"]),
            "conv_dict": {k: d[k] for k in d.files if k.startswith("conv_")},
        }


def baseline_orbits(path: str, species, device="cuda"):
    """(n, 9, N) device tensor of the listed species' orbits from a forward
    run's NPZ (the adjoint's FCT baseline read, adjoint.py:548-565): rows
    found through ``orbit_species_order`` (identity when absent)."""
    import torch
    with np.load(path, allow_pickle=False) as d:
        if "c_orbit" not in d.files:
            raise RuntimeError("the FCT baseline needs the orbit field c_orbit in the orbit NPZ")
        c = d["c_orbit"]
        order = list(d["orbit_species_order"].ravel()) if "orbit_species_order" in d.files \
            else list(range(c.shape[0]))
        row = {int(s): i for i, s in enumerate(order)}
        missing = [s for s in species if int(s) not in row]
        if missing:
            raise KeyError(f"species {missing} not in the orbit NPZ")
        return torch.as_tensor(np.stack([c[row[int(s)]] for s in species]), device=device)
