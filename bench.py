#!/usr/bin/env python
"""Benchmark: periodic orbits per second on B200 (one JSON line on rank 0).

Workload (per GPU, per step): one batch of 12 species orbits on an 80x72x15
domain (86,400 cells, 8 diurnal bins of 3 h) — one met draw of the
12-species x 12-draw batched workload; successive steps cycle through
different met draws.  A step is the whole hot path for the batch: transport
assembly of the 8 bins (K1), 96 numeric factorizations of I + dtau L (K3), and
the batched periodic-orbit GMRES over the chained bin solves (K4/K5) to tol
1e-8.  Headline ``value``: mixed precision (FP32 factors and solves, FP64
refinement, FP64 Arnoldi), all 12 orbits in one batch, inputs resident in HBM.
``e2e``: the same with every step's inputs copied from pinned host memory and
its orbits copied back inside the timed region (on a copy stream, double
buffered: step k+1's inputs and step k's orbits move while step k+1 computes).  ``plain_fp64``: the FP64 drop-in
solving the same orbits one at a time.  Inputs are seeded synthetic fields
(the reference's real met archive is not available).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun); orbits are independent, so each
rank solves its own batches (weak scaling); the only collectives are the
timing barrier and the max-over-ranks of the elapsed time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NZ, NY, NX = 15, 72, 80
N_SPECIES = 12
TOL = 1e-8
METRIC = "orbits/s at <=1e-6 rel err (mixed FP32/FP64, batched)"
WORKLOAD = "12 species x met draws, 80x72x15 (86,400 cells), 8 bins, GMRES(30) tol 1e-8, factor+solve"


def _env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic():
    """Per-launch DRAM traffic of the chain kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "k_chain_traffic.txt")
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_orbit_bin:"):
                    return float(line.split(":", 1)[1])
    except Exception:
        pass
    return None


class Clocks:
    def __init__(self, idx):
        self.idx = idx
        self.proc = None
        self.path = os.path.join("/tmp", f"orbit_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    sm.append(float(parts[0]))
                    mx = max(mx, float(parts[1]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _make_inputs(rank, n_draws, seed=2024):
    from orbit_b200 import synthetic
    from orbit_b200.shard import met_draw_seed
    mets = [synthetic.make_met(met_draw_seed(seed, rank, d), NZ, NY, NX, cmfmc_frac=0.3)
            for d in range(n_draws)]
    spc = [synthetic.make_species(seed + 17 + s, NZ, NY, NX) for s in range(N_SPECIES)]
    sinks = [[s.sink_diag(met) for s in spc] for met in mets]  # [draw][species] (8, N)
    emis = np.stack([s.emis for s in spc])  # (S, 8, N)
    return mets, spc, sinks, emis


def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _oracle_factors(met, sink, threads):
    """The 8 bin factorizations of one orbit (SuperLU COLAMD), one per host thread."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import assembly, orbit as oorbit
    Ts = [assembly.transport_block(g) for g in met]
    with ThreadPoolExecutor(max_workers=min(threads, 8)) as ex:
        return list(ex.map(lambda t: oorbit.factor_one_bin(assembly.species_operator(Ts[t], sink[t])),
                           range(8)))


def cpu_baseline_sample(met, spc, gpu_orbits):
    """The oracle port (SuperLU COLAMD + the reference's GMRES driver) on one
    orbit of the same workload (species 0 of the first met draw): its 8 bin
    factorizations on the host threads and the GMRES at the benchmark's tol,
    timed.  The same factors then continue the GMRES to tol 1e-12 (untimed),
    the truth against which the device orbits of that species are checked:
    max over cells and bins of |c - c_oracle| / max |c_oracle|."""
    from oracle import orbit as oorbit
    threads = _host_threads()
    sink = spc[0].sink_diag(met)
    t0 = time.perf_counter()
    lus = _oracle_factors(met, sink, threads)
    tf = time.perf_counter() - t0
    t0 = time.perf_counter()
    orb, info = oorbit.solve_orbit_one_species(lus, list(spc[0].emis), tol=TOL)
    ts = time.perf_counter() - t0
    truth, tinfo = oorbit.solve_orbit_one_species(lus, list(spc[0].emis), c_warm=orb[0], tol=1e-12)
    truth = np.stack(truth)
    scale = np.abs(truth).max()
    errs = {k: float(np.abs(np.asarray(v) - truth).max() / scale) for k, v in gpu_orbits.items()}
    errs["oracle_at_bench_tol"] = float(np.abs(np.stack(orb) - truth).max() / scale)
    lunz = int(lus[0].nnz)
    del lus
    t_orbit = tf + ts
    cpu = {"value": 1.0 / t_orbit, "unit": "orbits/s", "cores": min(threads, 8), "kind": "port",
           "sample": (f"one orbit (species 0, first met draw): 8 SuperLU COLAMD bin factorizations on "
                      f"{min(threads, 8)} host threads ({tf:.1f} s, nnz(LU) {lunz} per bin) + the GMRES "
                      f"driver to tol {TOL:g} ({ts:.1f} s, {info['gmres_iters']} iterations)")}
    parity = {"truth": "oracle orbit at tol 1e-12 (species 0, first met draw)",
              "max_rel_err_vs_oracle": errs, "oracle_truth_residual": tinfo["residual"]}
    return cpu, parity


def run_reference(args, rank, world):
    """The reference's CPU algorithm (oracle port: SciPy SuperLU COLAMD + the
    GMRES(30) driver) on this workload, with every host thread.  One orbit's
    work is eight bin factorizations (one per thread) and one GMRES solve, so a
    step is one bin of an orbit: its factorization plus an eighth of that
    orbit's GMRES.  The K steps are run as whole orbits (K rounded up to a
    multiple of 8), which bounds the run to a few minutes at the default K."""
    if rank != 0:
        return
    from oracle import assembly, orbit as oorbit
    mets, spc, sinks, emis = _make_inputs(0, 1)
    met = mets[0]
    threads = _host_threads()
    n_orbits = max(1, (args.steps + 7) // 8)

    def warm_sample():
        # untimed warm-up: one bin factor + solve
        L = assembly.species_operator(assembly.transport_block(met[0]), sinks[0][0][0])
        lu = oorbit.factor_one_bin(L)
        lu.solve(np.ones(L.shape[0]))

    for _ in range(max(0, min(args.warmup, 1))):
        warm_sample()
    t0 = time.perf_counter()
    for k in range(n_orbits):
        s = k % N_SPECIES
        lus = _oracle_factors(met, sinks[0][s], threads)
        oorbit.solve_orbit_one_species(lus, list(emis[s]), tol=TOL)
        del lus
    total = time.perf_counter() - t0
    v = n_orbits / total
    bins = 8 * n_orbits
    line = {"metric": METRIC, "value": v, "unit": "orbits/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / bins * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "step": "one bin of an orbit (factorization + 1/8 of its GMRES)",
                       "orbits_timed": n_orbits},
            "cpu_baseline": {"value": v, "unit": "orbits/s", "cores": min(threads, 8), "kind": "port",
                             "sample": f"{args.steps} bin steps rounded up to {n_orbits} whole orbits "
                                       f"({bins} bins): each orbit's 8 SuperLU (COLAMD) factorizations on "
                                       f"{min(threads, 8)} host threads + the reference GMRES driver "
                                       f"to tol {TOL:g}"},
            "e2e": {"value": v, "unit": "orbits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--draws", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-shared", action="store_true")
    ap.add_argument("--no-fct", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=200)
    args = ap.parse_args()
    rank, world, local = _env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from orbit_b200 import device
    from orbit_b200.symbolic import Symbolic

    mets, spc, sinks_h, emis_h = _make_inputs(rank, args.draws)
    sym = Symbolic.tuned(NZ, NY, NX, args.precision, N_SPECIES)  # autotuner's options, if cached
    # device-resident inputs
    met_dev = [[device.MetDevice(g) for g in met] for met in mets]
    sinks_d = [[torch.as_tensor(sinks_h[d][s], device="cuda") for s in range(N_SPECIES)]
               for d in range(args.draws)]
    E = torch.as_tensor(emis_h, device="cuda")
    fb = device.FactorBatch(sym, N_SPECIES, args.precision)

    def step(d, fbx=None, E_=None, sink_rows=None, mets_=None):
        fbx = fbx or fb
        mets_ = mets_ or met_dev[d]
        T = [device.assemble_transport(m) for m in mets_]
        sk = sink_rows if sink_rows is not None else sinks_d[d]
        fbx.numeric([T[b] for s in range(N_SPECIES) for b in range(8)],
                    [sk[s][b] for s in range(N_SPECIES) for b in range(8)])
        return fbx.solve(E if E_ is None else E_, tol=TOL)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for w in range(args.warmup):
        step(w % args.draws)
    # accuracy of the mixed path against the FP64 path on the same batch (untimed)
    err = None
    gpu_orbits = {}
    if args.precision == 32:
        orb32, _ = step(0)
        fb64 = device.FactorBatch(sym, N_SPECIES, 64)
        orb64, _ = step(0, fbx=fb64)
        err = float(((orb32 - orb64).abs().amax(dim=(1, 2)) / orb64.abs().amax(dim=(1, 2))).max())
        gpu_orbits["mixed_batched"] = orb32[0].cpu().numpy()
        gpu_orbits["fp64_batched"] = orb64[0].cpu().numpy()
        del fb64, orb64, orb32
        torch.cuda.empty_cache()

    # ---- timed: device-resident ----
    clocks = Clocks(local)
    fb.profile(1)
    launches0 = device.kernel_launches()
    barrier()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    lat = []
    infos = []
    for k in range(args.steps):
        e_a = torch.cuda.Event(enable_timing=True)
        e_b = torch.cuda.Event(enable_timing=True)
        e_a.record()
        _, info = step(k % args.draws)
        e_b.record()
        lat.append((e_a, e_b))
        infos.append(info)
    ev1.record()
    barrier()
    clk = clocks.stop()
    launches = device.kernel_launches() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    prof = fb.profile(2)
    fb.profile(0)
    lat_ms = sorted(a.elapsed_time(b) for a, b in lat)
    orbits = N_SPECIES * args.steps * world
    value = orbits / (ms / 1e3)

    # ---- solve only: the last step's factors resident, the batch solved again ----
    barrier()
    ev4 = torch.cuda.Event(enable_timing=True)
    ev5 = torch.cuda.Event(enable_timing=True)
    ev4.record()
    for k in range(args.steps):
        fb.solve(E, tol=TOL)
    ev5.record()
    barrier()
    ms_solve = max_over_ranks(ev4.elapsed_time(ev5))
    solve_only = {"value": orbits / (ms_solve / 1e3), "unit": "orbits/s", "ms_per_batch": ms_solve / args.steps}

    # ---- timed: end to end from pinned host buffers ----
    # one pinned host block and one device block per met draw, the device
    # fields re-pointed into it, so that a step's met input is one copy
    flat_pin, flat_dev = [], []
    for d, met in enumerate(mets):
        parts = [m.t[k].cpu().numpy().reshape(-1) for m in met_dev[d] for k in list(m.t.keys())]
        hp = torch.from_numpy(np.concatenate(parts)).pin_memory()
        dv = torch.empty_like(hp, device="cuda")
        dv.copy_(hp)
        off = 0
        for m in met_dev[d]:
            for k in list(m.t.keys()):
                sz = m.t[k].numel()
                m.t[k] = dv[off:off + sz].view(m.t[k].shape)
                off += sz
            m.rebind()
        flat_pin.append(hp)
        flat_dev.append(dv)
    sinks_p = [torch.from_numpy(np.stack(sinks_h[d])).pin_memory() for d in range(args.draws)]
    emis_p = torch.from_numpy(emis_h).pin_memory()
    # Inputs and results move on a copy stream, double-buffered, so that step
    # k+1's inputs arrive and step k's orbits leave while step k+1 computes;
    # every copy of every step lies inside the timed region (the copy stream
    # starts after the opening event and the closing event waits for its last
    # copy).  Step k+1 reads the met fields of draw (k+1) mod draws, which no
    # running step uses.
    out_p = [torch.empty((N_SPECIES, 9, sym.N), dtype=torch.float64).pin_memory() for _ in range(2)]
    dev_sinks = [torch.empty((N_SPECIES, 8, sym.N), dtype=torch.float64, device="cuda") for _ in range(2)]
    dev_E = [torch.empty_like(E) for _ in range(2)]
    h2d = flat_pin[0].numel() * 8 + sinks_p[0].numel() * 8 + emis_p.numel() * 8
    d2h = out_p[0].numel() * 8
    # two created streams: work on the legacy default stream would wait for
    # the copy stream and serialise the pipeline
    comp = torch.cuda.Stream()
    copy_st = torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]

    def enqueue_inputs(k):
        d, j = k % args.draws, k % 2
        with torch.cuda.stream(copy_st):
            flat_dev[d].copy_(flat_pin[d], non_blocking=True)
            dev_sinks[j].copy_(sinks_p[d], non_blocking=True)
            dev_E[j].copy_(emis_p, non_blocking=True)
            ev_in[j].record(copy_st)

    barrier()
    ev2 = torch.cuda.Event(enable_timing=True)
    ev3 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(comp):
        ev2.record(comp)
        copy_st.wait_event(ev2)
        enqueue_inputs(0)
        for k in range(args.steps):
            d, j = k % args.draws, k % 2
            if k + 1 < args.steps:
                enqueue_inputs(k + 1)
            comp.wait_event(ev_in[j])
            orb, _ = step(d, E_=dev_E[j], sink_rows=[[dev_sinks[j][s, b] for b in range(8)] for s in range(N_SPECIES)])
            done = torch.cuda.Event()
            done.record(comp)
            copy_st.wait_event(done)
            with torch.cuda.stream(copy_st):
                out_p[j].copy_(orb, non_blocking=True)
            orb.record_stream(copy_st)
        comp.wait_stream(copy_st)
        ev3.record(comp)
    barrier()
    ms_e2e = max_over_ranks(ev2.elapsed_time(ev3))
    e2e = {"value": orbits / (ms_e2e / 1e3), "unit": "orbits/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h)}

    # ---- plain FP64 drop-in, one orbit at a time (untimed by the headline) ----
    plain = None
    if not args.no_plain:
        # the FP64 drop-in with its own autotuned analysis (FP64, one orbit at a time)
        sym64 = Symbolic.tuned(NZ, NY, NX, 64, 1)
        fb1 = device.FactorBatch(sym64, 1, 64)
        times = []
        for s in range(N_SPECIES):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            T = [device.assemble_transport(m) for m in met_dev[0]]
            torch.cuda.synchronize()
            a.record()
            T = [device.assemble_transport(m) for m in met_dev[0]]
            fb1.numeric(T, [sinks_d[0][s][bb] for bb in range(8)])
            o1, i1 = fb1.solve(E[s:s + 1], tol=TOL)
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
            if s == 0:
                gpu_orbits["fp64_plain"] = o1[0].cpu().numpy()
        plain = {"value": 1e3 * len(times) / sum(times), "unit": "orbits/s",
                 "latency_ms_p50": float(np.percentile(times, 50)),
                 "latency_ms_p99": float(np.percentile(times, 99)),
                 "tuning": sym64.options}
        del fb1

    # ---- shared operator: 64 marginal right-hand sides and 64 adjoint receptors
    # on one factor set (species 0, draw 0), FP32 factors, tol 1e-6 ----
    shared = None
    if not args.no_shared:
        n_rhs, stol = 64, 1e-6
        fbS = device.FactorBatch(sym, n_rhs, args.precision, n_sets=1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        T0 = [device.assemble_transport(m) for m in met_dev[0]]
        a.record()
        fbS.numeric(T0, [sinks_d[0][0][bb] for bb in range(8)])
        b.record()
        torch.cuda.synchronize()
        t_fac = a.elapsed_time(b)
        rng = np.random.default_rng(2027)
        dE = np.zeros((n_rhs, 8, sym.N))
        R = np.zeros((n_rhs, 8, sym.N))
        e0 = emis_h[0].reshape(8, NZ, NY, NX)
        for q in range(n_rhs):
            j0, i0 = rng.integers(0, NY - 5), rng.integers(0, NX - 5)
            scale = np.exp(rng.normal(0.0, 0.1)) - 1.0  # +-10 % lognormal scaling of the patch
            d = np.zeros((8, NZ, NY, NX))
            d[:, 0, j0:j0 + 5, i0:i0 + 5] = scale * e0[:, 0, j0:j0 + 5, i0:i0 + 5]
            dE[q] = d.reshape(8, -1)
            j1, i1 = rng.integers(0, NY - 5), rng.integers(0, NX - 5)
            r = np.zeros((8, NZ, NY, NX))
            r[:, 0, j1:j1 + 5, i1:i1 + 5] = 1.0 / (8 * 25)  # receptor: mean over a surface patch
            R[q] = r.reshape(8, -1)
        dE_d = torch.as_tensor(dE, device="cuda")
        R_d = torch.as_tensor(R, device="cuda")
        fbS.solve(dE_d, tol=stol)
        fbS.solve_adjoint(R_d, tol=stol)
        barrier()
        a.record()
        _, inf_f = fbS.solve(dE_d, tol=stol)
        b.record()
        barrier()
        t_f = a.elapsed_time(b)
        a.record()
        _, inf_a = fbS.solve_adjoint(R_d, tol=stol)
        b.record()
        barrier()
        t_a = a.elapsed_time(b)
        shared = {"rhs": n_rhs, "tol": stol, "factor_ms": t_fac,
                  "forward_orbits_per_s": 1e3 * n_rhs / t_f, "adjoint_orbits_per_s": 1e3 * n_rhs / t_a,
                  "forward_ms": t_f, "adjoint_ms": t_a,
                  "chains_forward": float(np.median(inf_f[:, 7])), "chains_adjoint": float(np.median(inf_a[:, 7])),
                  "all_converged": bool(np.all(inf_f[:, 4] > 0) and np.all(inf_a[:, 4] > 0))}
        del fbS

    # ---- the full-domain configuration with the FCT correction on: pass 0
    # without FCT, then 6 deferred-correction passes (each a warm-started
    # solve whose forcing adds the limited anti-diffusive source of the
    # previous pass), for the mixed batch of 12 and the plain FP64 drop-in
    # one orbit at a time; factorization included ----
    fct = None
    if not args.no_fct:
        from orbit_b200 import api
        passes = 6
        d0 = 0
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        a.record()
        T = [device.assemble_transport(m) for m in met_dev[d0]]
        fb.numeric([T[bb] for s in range(N_SPECIES) for bb in range(8)],
                   [sinks_d[d0][s][bb] for s in range(N_SPECIES) for bb in range(8)])
        _, infs = api.solve_with_fct(fb, met_dev[d0], E, passes, tol=TOL)
        b.record()
        barrier()
        t_mixed = a.elapsed_time(b)
        fct = {"passes": passes, "tol": TOL, "mixed_batched_orbits_per_s": 1e3 * N_SPECIES / t_mixed,
               "mixed_batched_ms": t_mixed,
               "all_converged": bool(all(np.all(i[:, 4] > 0) for i in infs)),
               "chains_per_pass_mixed": [float(np.median(i[:, 7])) for i in infs]}
        if not args.no_plain:
            sym64 = Symbolic.tuned(NZ, NY, NX, 64, 1)
            fbp = device.FactorBatch(sym64, 1, 64)
            tp = []
            for s in range(2):  # two orbits of the plain drop-in
                barrier()
                a.record()
                T = [device.assemble_transport(m) for m in met_dev[d0]]
                fbp.numeric(T, [sinks_d[d0][s][bb] for bb in range(8)])
                _, infp = api.solve_with_fct(fbp, met_dev[d0], E[s:s + 1], passes, tol=TOL)
                b.record()
                barrier()
                tp.append(a.elapsed_time(b))
            fbp.close()
            fct["plain_fp64_orbits_per_s"] = 1e3 * len(tp) / sum(tp)
            fct["chains_per_pass_plain"] = [float(i[0, 7]) for i in infp]
            fct["mixed_vs_plain"] = fct["mixed_batched_orbits_per_s"] / fct["plain_fp64_orbits_per_s"]

    # ---- roofline of the chained-solve kernel (K4) ----
    peak, peak_kind = _peaks()
    chain_ms_avg = prof["chain_ms"] / max(prof["chain_launches"], 1)
    chain_bytes = prof["chain_bytes"] / max(prof["chain_launches"], 1)
    achieved = chain_bytes / (chain_ms_avg * 1e-3) / 1e9 if chain_ms_avg > 0 else 0.0
    vb = 4 if args.precision == 32 else 8
    tr = _profile_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (tr * chain_bytes / (sym.lunz * vb)) if tr else None,
                "kernel": "k_chain", "algorithmic_bytes_per_launch": chain_bytes,
                "avg_launch_ms": chain_ms_avg, "launches": prof["chain_launches"],
                "factor_nnz_per_bin": sym.lunz}
    factor = {"kernel_group": "numeric factorization (K3)",
              "ms_per_step": prof["factor_ms"] / max(args.steps, 1),
              "achieved_tflops": prof["factor_flops"] / (prof["factor_ms"] * 1e-3) / 1e12
              if prof["factor_ms"] > 0 else None,
              "flops_per_factor": sym.info["factor_flops"]}

    # ---- serving: a Poisson stream of forward / marginal / adjoint requests on
    # four domain sizes under the 150 GB admission budget (the batch's own
    # device buffers released first) ----
    serving = None
    if not args.no_serving and world == 1:
        from orbit_b200 import serve_bench
        fb.close()
        torch.cuda.empty_cache()
        serving = serve_bench.run(requests=args.serve_requests, rate=200.0, budget_gb=150.0)
        # the same mix at a rate one GPU sustains (about a quarter of its
        # throughput), where the latencies are service times, not queueing
        light = serve_bench.run(requests=max(8, args.serve_requests // 5), rate=5.0, budget_gb=150.0, seed=6)
        serving["light_load"] = {"arrival_rate_per_s": 5.0, "requests": light["requests"], "value": light["value"],
                                 "latency_ms": light["latency_ms"], "all_converged": light["all_converged"]}

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, parity = cpu_baseline_sample(mets[0], spc, gpu_orbits)

    if rank == 0:
        it = [r[0] for inf in infos for r in inf]
        line = {
            "metric": METRIC, "value": value, "unit": "orbits/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == 32 else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "orbits_per_step_per_gpu": N_SPECIES,
                       "met_draws": args.draws, "grid": [NZ, NY, NX], "tol": TOL,
                       "precision": "fp32 factors + fp64 refinement" if args.precision == 32 else "fp64",
                       "l2": "inputs and factors (>15 GB) exceed L2 each step", "parallelism": f"orbits x{world}",
                       "tuning": sym.options},
            "e2e": e2e, "solve_only": solve_only, "roofline": roofline, "factorization": factor,
            "cpu_baseline": cpu,
            "clocks": clk, "gpu_launches": int(launches),
            "latency_ms": {"batch_p50": float(np.percentile(lat_ms, 50)),
                           "batch_p99": float(np.percentile(lat_ms, 99))},
            "plain_fp64": plain,
            "shared_operator": shared,
            "fct_config": fct,
            "serving": serving,
            "mixed_vs_plain": (value / world / plain["value"]) if plain else None,
            "max_rel_err_vs_fp64": err,
            "parity": parity,
            "gmres_iters_median": float(np.median(it)) if it else None,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
