"""Golden digest of the reference's own orbits on the 80x72x15 benchmark workload.

Run where the reference checkout is importable (its default location is used
unless ORBIT_REFERENCE is set):

    python tests/golden/make_bench_golden.py

It builds the first met draw of the 12-species benchmark (80x72x15, 86,400
cells, convective mass flux in 30 % of the columns; the same seeds as
``bench.py``), and for species 0 and 1 runs the reference's
``_factor_one_bin`` (SciPy SuperLU, its no-UMFPACK path) on the eight bins in
parallel threads and ``solve_orbit_one_species`` at tol 1e-12.  A full orbit
is 9 x 86,400 doubles per species, too large to commit, so the file keeps a
digest: the values at 16,384 fixed random (bin, cell) positions, every bin's
max |c| and L2 norm, the GMRES info, and the reference's mass-balance
statistics of the eight bins (the gate's input).  The GPU tests compare their
orbits with it; nothing reads the reference at test time.
"""
from __future__ import annotations

import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)
sys.path.insert(0, os.environ.get("ORBIT_REFERENCE", "/root/reference"))

import scipy.sparse as sp  # noqa: E402

from orbit.core.indexing import CellIndexer  # noqa: E402
from orbit.core import operator  # noqa: E402
from orbit.core.orbit import _factor_one_bin, solve_orbit_one_species, DTAU, N_BINS  # noqa: E402

from make_golden import to_griddata  # noqa: E402
from orbit_b200 import synthetic  # noqa: E402
from orbit_b200.shard import met_draw_seed  # noqa: E402

NZ, NY, NX = 15, 72, 80
SEED = 2024          # bench.py's base seed
N_SAMPLE = 16384
SPECIES = (0, 1)


def bench_inputs():
    """The benchmark's first met draw and its species (bench.py::_make_inputs)."""
    met = synthetic.make_met(met_draw_seed(SEED, 0, 0), NZ, NY, NX, cmfmc_frac=0.3)
    spc = [synthetic.make_species(SEED + 17 + s, NZ, NY, NX) for s in range(max(SPECIES) + 1)]
    return met, spc


def sample_positions(N):
    rng = np.random.default_rng(99)
    return rng.integers(0, (N_BINS + 1) * N, size=N_SAMPLE).astype(np.int64)


def main():
    met, spc = bench_inputs()
    idx = CellIndexer(NZ, NY, NX)
    N = idx.N
    grids = [to_griddata(m) for m in met]
    t0 = time.time()
    T = [operator.assemble_transport_block(g, idx) for g in grids]
    mb = operator.mass_balance_diagnostics(grids, idx)
    print(f"assembly + mass balance {time.time() - t0:.1f}s", flush=True)
    I_N = sp.eye(N, format="csc")
    pos = sample_positions(N)
    out = {"pos": pos, "grid": np.array([NZ, NY, NX]), "species": np.array(SPECIES)}
    keys = ["interior_median", "interior_p90", "interior_p99", "interior_max", "top_median", "top_p90"]
    out["mb_keys"] = np.array(keys)
    out["mb_vals"] = np.array([mb[k] for k in keys])
    for s in SPECIES:
        d = spc[s].sink_diag(met)
        L = [(T[t] + sp.diags(d[t])).tocsc() for t in range(N_BINS)]
        t0 = time.time()
        with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
            lus = list(ex.map(lambda t: _factor_one_bin(L[t], I_N, None, None), range(N_BINS)))
        tf = time.time() - t0
        t0 = time.time()
        orbit, info = solve_orbit_one_species(lus, list(spc[s].emis), DTAU, tol=1e-12, maxiter=200)
        ts = time.time() - t0
        C = np.stack(orbit)
        print(f"species {s}: factor {tf:.1f}s, solve {ts:.1f}s, iters {info['gmres_iters']}, "
              f"residual {info['residual']:.2e}", flush=True)
        out[f"s{s}_vals"] = C.reshape(-1)[pos]
        out[f"s{s}_max"] = np.abs(C).max(axis=1)
        out[f"s{s}_norm"] = np.linalg.norm(C, axis=1)
        out[f"s{s}_info"] = np.array([info["gmres_iters"], info["residual"], info["periodicity"],
                                      info["neg_frac"]])
        del lus
    path = os.path.join(HERE, "bench_grid_digest.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
