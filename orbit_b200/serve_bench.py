"""Serving benchmark: a Poisson stream of orbit requests on mixed domains.

    python -m orbit_b200.serve_bench [--requests 200] [--rate 200] [--budget-gb 150]

Requests arrive at `rate` per second (exponential inter-arrival times); each
picks a domain uniformly from 24x20, 40x36, 60x54 and 80x72 (15 layers), a
met month, a kind (60 % forward, 30 % marginal, 10 % adjoint) and 1-12
right-hand sides (forward: species; marginal: emission perturbations of one
species; adjoint: receptors); factors are cached per (domain, month) under
the HBM budget.  Prints one JSON line: orbits/s, p50/p99 request latency
(arrival to completion), batches, peak admitted bytes.  Inputs are seeded
synthetic fields.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import synthetic
from .serve import OrbitRequest, OrbitServer

DOMAINS = [(15, 20, 24), (15, 36, 40), (15, 54, 60), (15, 72, 80)]
N_SPECIES = 12


def make_provider(seed=2024):
    cache = {}

    def provider(domain, month):
        key = (domain, month)
        if key not in cache:
            nz, ny, nx = domain
            mets = synthetic.make_met(seed + 7919 * month + ny * 131 + nx, nz, ny, nx, cmfmc_frac=0.3)
            spc = [synthetic.make_species(seed + 17 + s, nz, ny, nx) for s in range(N_SPECIES)]
            cache[key] = (mets, [s.sink_diag(mets) for s in spc], spc)
        mets, sinks, _ = cache[key]
        return mets, sinks

    def species(domain, month):
        provider(domain, month)
        return cache[(domain, month)][2]

    return provider, species


def make_requests(n, rate, months, rng, species_of):
    """Poisson arrivals; forward requests solve 1-12 species' emissions, marginal
    requests 1-12 emission perturbations of one species on its (shared)
    operator (+-10 % lognormal scaling of random 5x5 surface patches, the
    marginal configuration), adjoint requests 1-12 receptors (patch means)."""
    reqs = []
    t = 0.0
    for _ in range(n):
        t += rng.exponential(1.0 / rate)
        domain = DOMAINS[rng.integers(len(DOMAINS))]
        month = int(rng.integers(months))
        u = rng.random()
        kind = "forward" if u < 0.6 else ("marginal" if u < 0.9 else "adjoint")
        k = int(rng.integers(1, N_SPECIES + 1))
        fields = species_of(domain, month)
        nz, ny, nx = domain
        N = nz * ny * nx
        if kind == "forward":
            sp = sorted(rng.choice(N_SPECIES, size=k, replace=False).tolist())
            F = np.stack([fields[s].emis for s in sp])
        else:
            s0 = int(rng.integers(N_SPECIES))
            sp = [s0] * k
            F = np.zeros((k, 8, nz, ny, nx))
            for q in range(k):
                j0, i0 = rng.integers(0, ny - 5), rng.integers(0, nx - 5)
                if kind == "marginal":
                    e0 = fields[s0].emis.reshape(8, nz, ny, nx)
                    scale = np.exp(rng.normal(0.0, 0.1)) - 1.0
                    F[q, :, 0, j0:j0 + 5, i0:i0 + 5] = scale * e0[:, 0, j0:j0 + 5, i0:i0 + 5]
                else:
                    F[q, :, 0, j0:j0 + 5, i0:i0 + 5] = 1.0 / (8 * 25)
            F = F.reshape(k, 8, N)
        reqs.append((t, OrbitRequest(domain=domain, month=month, kind=kind, species=sp, forcing=F, tol=1e-6)))
    return reqs


def run(requests=200, rate=200.0, months=2, budget_gb=150.0, slots=24, workers=2, seed=5):
    """Serve one seeded Poisson stream; returns the measured record."""
    rng = np.random.default_rng(seed)
    provider, species_of = make_provider()
    reqs = make_requests(requests, rate, months, rng, species_of)
    for domain in DOMAINS:  # inputs generated before the clock starts
        for month in range(months):
            provider(domain, month)
    srv = OrbitServer(provider, hbm_budget_bytes=budget_gb * 1e9, slots=slots, workers=workers).start()
    t0 = time.perf_counter()
    peak = 0.0
    for t_arr, r in reqs:
        while time.perf_counter() - t0 < t_arr:
            time.sleep(0.0005)
        srv.submit(r)
        peak = max(peak, srv.used_bytes())
    for _, r in reqs:
        r.done.wait()
        peak = max(peak, srv.used_bytes())
    wall = time.perf_counter() - t0
    srv.stop()
    lat = np.array([r.latency for _, r in reqs]) * 1e3
    errs = [r.error for _, r in reqs if r.error]
    n_orb = sum(len(r.species) for _, r in reqs)
    kinds = {k: sum(1 for _, r in reqs if r.kind == k) for k in ("forward", "marginal", "adjoint")}
    conv = all(r.info is not None and bool(np.all(r.info[:, 4] > 0)) for _, r in reqs if not r.error)
    return {
        "metric": "served orbits/s (Poisson arrivals, mixed domains)", "value": n_orb / wall,
        "unit": "orbits/s", "requests": len(reqs), "orbits": n_orb, "wall_s": wall,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "batches": srv.batches, "peak_admitted_gb": peak / 1e9, "budget_gb": budget_gb,
        "kinds": kinds, "all_converged": conv, "errors": errs[:3], "arrival_rate_per_s": rate,
        "domains": [f"{nx}x{ny}x{nz}" for nz, ny, nx in DOMAINS], "tol": 1e-6, "precision": "fp32+fp64"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--months", type=int, default=2)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--slots", type=int, default=24)
    ap.add_argument("--workers", type=int, default=2)
    ap.add_argument("--seed", type=int, default=5)
    args = ap.parse_args()
    print(json.dumps(run(args.requests, args.rate, args.months, args.budget_gb, args.slots, args.workers,
                         args.seed)))


if __name__ == "__main__":
    main()
