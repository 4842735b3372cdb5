"""Small, fixed device workloads for profiling the kernels one at a time.

    python -m orbit_b200.profile_cases chain  --precision 32 --orbits 12
    python -m orbit_b200.profile_cases factor --precision 32 --orbits 12
    python -m orbit_b200.profile_cases solve  --precision 32 --orbits 12

Each builds the 80x72x15 workload (seeded synthetic met, 12 species), factors
it, and then runs the named stage: three chained-solve launches over all
orbits and 8 bins (chain), nothing more (factor), or one batched GMRES solve
(solve).  Shapes can be reduced with --grid nz ny nx for small captures.
"""
from __future__ import annotations

import argparse

import torch

from . import device, synthetic
from .symbolic import Symbolic


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("stage", choices=["chain", "factor", "solve"])
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--orbits", type=int, default=12)
    ap.add_argument("--grid", type=int, nargs=3, default=[15, 72, 80])
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args()
    nz, ny, nx = args.grid
    met = synthetic.make_met(2024, nz, ny, nx, cmfmc_frac=0.3)
    spc = [synthetic.make_species(2041 + s, nz, ny, nx) for s in range(args.orbits)]
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(d, device="cuda") for s in spc for d in s.sink_diag(met)]
    sym = Symbolic.tuned(nz, ny, nx, args.precision, args.orbits)  # the bench's analysis options
    fb = device.FactorBatch(sym, args.orbits, args.precision)
    fb.numeric([T[t] for _ in range(args.orbits) for t in range(8)], sinks)
    if args.stage == "chain":
        x = torch.randn(args.orbits, sym.N, device="cuda", dtype=torch.float64)
        for _ in range(args.repeat):
            fb.chain(x, refine=False)
    elif args.stage == "solve":
        E = torch.stack([torch.as_tensor(s.emis, device="cuda") for s in spc])
        fb.solve(E, tol=1e-8)
    torch.cuda.synchronize()
    print(f"{args.stage} done: N={sym.N} factor nnz/bin={sym.lunz}")


if __name__ == "__main__":
    main()
