"""Autotuner for the symbolic analysis' tuning options.

The options that shape the launches (nested-dissection leaf size, solve row
chunk size, tensor-core supernode threshold, whole-subtree solve-task
divisor; see ``orbit_symbolic_create_ex``) trade latency against per-task
overhead differently for each grid shape, precision and batch width.  The
tuner measures candidates on the device with the workload they serve: one
numeric factorization of ``batch`` orbits (8 bins each) and one batched
periodic-orbit solve, seeded synthetic inputs of the requested shape.  It
walks the options one at a time (coordinate descent from the defaults), keeps
the fastest, and records the result in a JSON cache keyed by device name,
shape, precision and batch width.

    python -m orbit_b200.autotune --grid 15 72 80 --precision 32 --batch 12 --write

``tuned_options`` reads the cache (``ORBIT_B200_TUNE_CACHE`` or the
package's ``tuned.json``); ``Symbolic.tuned`` builds an analysis with them.
"""
from __future__ import annotations

import argparse
import json
import os
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

DEFAULTS = {"leaf_cells": 64, "chunk_elems": 8192, "tc_min_n": 48, "subtree_div": 0}
SPACE = {
    "leaf_cells": [48, 64, 80, 96],
    "chunk_elems": [4096, 8192, 16384],
    "tc_min_n": [32, 48, 96],
    "subtree_div": [0, 1024],
}
_HERE = os.path.dirname(os.path.abspath(__file__))


def cache_path() -> str:
    return os.environ.get("ORBIT_B200_TUNE_CACHE", os.path.join(_HERE, "tuned.json"))


def _key(device: str, shape: Sequence[int], precision: int, batch: int) -> str:
    nz, ny, nx = shape
    return f"{device}|{nz}x{ny}x{nx}|fp{precision}|b{batch}"


def load_cache(path: Optional[str] = None) -> Dict:
    path = path or cache_path()
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def tuned_options(shape: Sequence[int], precision: int, batch: int, device: Optional[str] = None,
                  path: Optional[str] = None) -> Dict[str, int]:
    """Cached options for this device, shape and precision at the nearest tuned
    batch width; the defaults when nothing matches."""
    if device is None:
        import torch
        device = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    cache = load_cache(path)
    nz, ny, nx = shape
    best, best_d = None, None
    prefix = f"{device}|{nz}x{ny}x{nx}|fp{precision}|b"
    for k, v in cache.items():
        if not k.startswith(prefix):
            continue
        d = abs(int(k[len(prefix):]) - batch)
        if best_d is None or d < best_d:
            best, best_d = v, d
    return dict(best["options"]) if best else dict(DEFAULTS)


def _workload(shape, batch, seed=2024):
    import torch
    from . import device as dev, synthetic
    nz, ny, nx = shape
    met = synthetic.make_met(seed, nz, ny, nx, cmfmc_frac=0.3)
    spc = [synthetic.make_species(seed + 17 + s, nz, ny, nx) for s in range(batch)]
    mets = [dev.MetDevice(g) for g in met]
    T = [dev.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(d, device="cuda") for s in spc for d in s.sink_diag(met)]
    E = torch.as_tensor(np.stack([s.emis for s in spc]), device="cuda")
    return T, sinks, E


def measure(shape, precision, batch, options, reps=2, tol=1e-8, workload=None) -> float:
    """Median ms of one factorization plus one batched solve with these options."""
    import torch
    from . import device as dev
    from .symbolic import Symbolic
    T, sinks, E = workload or _workload(shape, batch)
    sym = Symbolic(*shape, **options)
    fb = dev.FactorBatch(sym, batch, precision)
    times = []
    try:
        for r in range(reps + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fb.numeric([T[t] for _ in range(batch) for t in range(8)], sinks)
            fb.solve(E, tol=tol)
            b.record()
            torch.cuda.synchronize()
            if r > 0:  # the first pass pays one-off set-up
                times.append(a.elapsed_time(b))
    finally:
        fb.close()
        sym.close()
        torch.cuda.empty_cache()
    return float(np.median(times))


def tune(shape, precision=32, batch=12, space=None, reps=2, log=print) -> Dict:
    """Coordinate descent over `space` from the defaults; returns the record
    stored in the cache (options, ms per batch, candidates measured)."""
    import torch
    space = space or SPACE
    wl = _workload(shape, batch)
    best = dict(DEFAULTS)
    tried: Dict[str, float] = {}

    def run(opts):
        k = json.dumps(opts, sort_keys=True)
        if k not in tried:
            tried[k] = measure(shape, precision, batch, opts, reps=reps, workload=wl)
            log(f"  {opts} -> {tried[k]:.1f} ms")
        return tried[k]

    best_ms = run(best)
    for name, values in space.items():
        for v in values:
            cand = dict(best)
            cand[name] = v
            ms = run(cand)
            if ms < best_ms:
                best, best_ms = cand, ms
    return {"options": best, "ms_per_batch": best_ms, "orbits_per_s": 1e3 * batch / best_ms,
            "default_ms": tried[json.dumps(DEFAULTS, sort_keys=True)],
            "candidates": len(tried), "device": torch.cuda.get_device_name(),
            "date": time.strftime("%Y-%m-%d")}


def main(argv: Optional[List[str]] = None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--grid", type=int, nargs=3, default=[15, 72, 80], metavar=("NZ", "NY", "NX"))
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--batch", type=int, default=12)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--write", action="store_true", help="store the result in the cache")
    ap.add_argument("--cache", default=None)
    args = ap.parse_args(argv)
    rec = tune(args.grid, args.precision, args.batch, reps=args.reps)
    print(json.dumps(rec), flush=True)
    if args.write:
        path = args.cache or cache_path()
        cache = load_cache(path)
        cache[_key(rec["device"], args.grid, args.precision, args.batch)] = rec
        with open(path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main()
