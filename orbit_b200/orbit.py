"""Drop-in for the reference's periodic-orbit solver (orbit/core/orbit.py).

Same names, signatures, return values and conventions as the reference:

* ``_factor_one_bin(L_s_tau, I_N, umfpack_sym, perm)`` (orbit.py:79-96)
  returns a ``DeviceLU`` for ``A = I + DTAU L``;
* ``apply_monodromy`` / ``compute_s`` (orbit.py:99-120) run the eight bin
  solves as one chained device launch;
* ``solve_orbit_one_species`` (orbit.py:123-210) factors the eight bins in
  one batch and runs the restarted GMRES on the device; it returns the orbit
  as nine host arrays and the info dict (``gmres_iters``, ``residual``,
  ``periodicity``, ``neg_frac``); non-convergence prints the reference's
  WARNING and returns (orbit.py:184-186);
* ``solve_orbit_all_species`` (orbit.py:468-806) solves the species wave by
  wave (sources before targets, the reference's DAG waves and K-couplings,
  zero-source skip, copy-verbatim skip, LU cache, seed orbits, end-of-bin
  couplings); all species of a wave are factored and solved in one batch.

There is no CPU fallback: every factorization and solve runs in
liborbit_b200 on the GPU.
"""
from __future__ import annotations

import time
import weakref
from typing import Dict, List, Optional, Sequence

import numpy as np

from .solve import DeviceLU, DeviceSymbolic, umfpack_symbolic
from .synthetic import DTAU, N_BINS

_SPECIES_NAMES = ["VBS_C100", "PM2.5", "NH", "SO2", "NOx", "pSO4", "TotalNO3",
                  "O3", "CO", "VBS_C10", "VBS_C1", "VBS_C01", "VBS_C1000", "POA"]
_SOLVE_ORDER = [0, 1, 13, 2, 3, 4, 5, 6, 7, 8, 12, 9, 10, 11]


def _factor_one_bin(L_s_tau, I_N, umfpack_sym, perm):
    """A_tau = I + L DTAU on the device (factored lazily, or batched with its bin set)."""
    if umfpack_sym is None:
        raise RuntimeError("the device path needs the symbolic handle from umfpack_symbolic")
    return DeviceLU(L_s_tau, umfpack_sym, dtau=DTAU)


# One 8-bin factor batch per list of DeviceLUs (keyed by the LU objects).
_batches: "weakref.WeakValueDictionary" = weakref.WeakValueDictionary()
_batch_refs: Dict[tuple, object] = {}


class _BinSet:
    """Eight DeviceLUs factored together (1 orbit x 8 bins)."""

    def __init__(self, lus: Sequence[DeviceLU]):
        from .device import FactorBatch
        sym = lus[0].sym
        if any(lu.sym is not sym for lu in lus) or len(lus) != N_BINS:
            raise ValueError("solve_orbit_one_species needs 8 DeviceLUs built on one symbolic")
        dtau = lus[0].dtau
        self.fb = FactorBatch(sym, 1, lus[0].precision)
        self.fb.numeric([lu.device_stencil() for lu in lus], None, dtau)
        self.N = sym.N
        for t, lu in enumerate(lus):  # each LU now solves through its bin of this batch
            lu.attach_to_set(self.fb, t)


def _bin_set(lu_list_8) -> _BinSet:
    lus = list(lu_list_8)
    if not all(isinstance(lu, DeviceLU) for lu in lus):
        raise TypeError("the device solver needs DeviceLU objects (from _factor_one_bin)")
    key = tuple(id(lu) for lu in lus)
    bs = _batch_refs.get(key)
    if bs is None:
        bs = _BinSet(lus)
        _batch_refs[key] = bs
        for lu in lus:  # drop the batch when any of its LUs goes away
            weakref.finalize(lu, _batch_refs.pop, key, None)
    return bs


def apply_monodromy(v, lu_list_8):
    """M v = P_8 ... P_1 v (orbit.py:99-107), one chained launch."""
    import torch
    bs = _bin_set(lu_list_8)
    x = torch.as_tensor(np.ascontiguousarray(v, dtype=np.float64), device="cuda")[None]
    return bs.fb.chain(x)[0].cpu().numpy()


def compute_s(lu_list_8, e_tau_list, dtau=DTAU):
    """One forward sweep from zero with emissions (orbit.py:110-120)."""
    import torch
    bs = _bin_set(lu_list_8)
    e = torch.as_tensor(np.stack([np.asarray(x, dtype=np.float64) for x in e_tau_list]), device="cuda")
    x = torch.zeros((1, bs.N), dtype=torch.float64, device="cuda")
    return bs.fb.chain(x, forcing=e[None], fscale=float(dtau))[0].cpu().numpy()


def _info_dict(row):
    return {"gmres_iters": int(row[0]), "residual": float(row[1]), "periodicity": float(row[2]),
            "neg_frac": float(row[3])}


def solve_orbit_one_species(lu_list_8, e_tau_list, dtau=DTAU, c_warm=None, tol=1e-6, maxiter=200):
    """GMRES(30) on (I - M) c_0 = s on the device (orbit.py:123-210)."""
    import torch
    bs = _bin_set(lu_list_8)
    e = torch.as_tensor(np.stack([np.asarray(x, dtype=np.float64) for x in e_tau_list]), device="cuda")
    w = None if c_warm is None else torch.as_tensor(np.asarray(c_warm, dtype=np.float64), device="cuda")
    orb, info = bs.fb.solve(e[None], c_warm=w, tol=tol, maxiter=maxiter, dtau=dtau)
    o = orb[0].cpu().numpy()
    return [o[t].copy() for t in range(N_BINS + 1)], _info_dict(info[0])


def _build_solve_waves(sources_for_target, solve_order, skip_species):
    """DAG waves (orbit.py:397-465): cyclic edges dropped, placement iterated to a fixpoint."""
    cyclic = set()
    for tgt, srcs in sources_for_target.items():
        for src in srcs:
            if tgt in sources_for_target.get(src, []):
                cyclic.add((tgt, src))
    eff = {t: [s for s in srcs if (t, s) not in cyclic] for t, srcs in sources_for_target.items()}
    placed = {}
    for _ in range(len(solve_order) + 2):
        changed = False
        for s in solve_order:
            if s in skip_species or not eff.get(s):
                new = 0
            else:
                new = max(placed.get(src, 0) for src in eff[s]) + 1
            if placed.get(s) != new:
                placed[s] = new
                changed = True
        if not changed:
            break
    waves = [[] for _ in range((max(placed.values()) if placed else 0) + 1)]
    for s in solve_order:
        waves[placed[s]].append(s)
    return waves


class SpeciesFactors:
    """LU-cache entry: the eight factorizations of one species inside a batch."""

    def __init__(self, fb, set_index):
        self.fb = fb
        self.set_index = set_index


def _emissions_for(emissions_SN, s, N):
    if emissions_SN.ndim == 1:
        return [emissions_SN[s * N:(s + 1) * N]] * N_BINS
    return [emissions_SN[t, s * N:(s + 1) * N] for t in range(N_BINS)]


def _diag_of(K, N):
    """The diagonal of a coupling block, which must be diagonal (every K block
    of assemble_species_operators is, operator.py:419-547)."""
    import scipy.sparse as sp
    C = sp.coo_matrix(K)
    if C.shape != (N, N):
        raise ValueError(f"coupling block has shape {C.shape}, expected ({N}, {N})")
    off = (C.row != C.col) & (C.data != 0)
    if np.any(off):
        raise ValueError("the device coupling takes diagonal K blocks only")
    d = np.zeros(N)
    np.add.at(d, C.row[C.row == C.col], C.data[C.row == C.col])
    return d


def solve_orbit_all_species(L_species_per_bin, K_sources_per_bin, emissions_SN, N, umfpack_sym=None,
                            perm=None, tol=1e-6, maxiter=200, verbose=True, c_warm_SN=None,
                            lu_cache=None, skip_solve_species=None, cached_orbits=None,
                            return_lu_cache=False, keep_lu_species=None,
                            extra_rhs_per_bin_per_species=None, seed_orbits=None, endbin_keys=None,
                            precision=64):
    """All species' periodic orbits, wave by wave, each wave one device batch.

    Arguments and result as in the reference (orbit.py:468-559).  ``umfpack_sym``
    may be omitted: the symbolic is then built from the first operator's
    pattern.  ``precision=32`` selects FP32 factors with FP64 refinement.
    Solved orbits stay on the device between waves: the coupled right-hand
    sides e_tau - K c_src[tau] (or c_src[tau + 1] for ``endbin_keys``,
    orbit.py:249-307) are formed there (``orbit_source_coupling``); the host
    receives the orbits once, at the end.
    """
    import torch
    from . import device
    from .device import FactorBatch

    n_species = len(L_species_per_bin[0])
    emissions_SN = np.asarray(emissions_SN, dtype=np.float64)
    if umfpack_sym is None:
        first = next((L for L in L_species_per_bin[0] if L is not None), None)
        if first is not None:
            umfpack_sym = umfpack_symbolic(first, verbose=verbose)
        elif lu_cache:
            umfpack_sym = next(iter(lu_cache.values())).fb.sym
        else:
            raise ValueError("no operator and no LU cache to take the symbolic analysis from; pass umfpack_sym")
    sym = umfpack_sym.sym if isinstance(umfpack_sym, DeviceSymbolic) else umfpack_sym
    dev_orbits = {}  # species -> (9, N) device tensor
    host_orbits = {}  # species -> list of host arrays (seeds and cached copies, returned as given)
    gmres_iters = np.zeros(n_species, dtype=int)
    gmres_resid = np.zeros(n_species)
    periodicity = np.zeros(n_species)
    if seed_orbits is not None:
        for s, orb in seed_orbits.items():
            host_orbits[s] = [np.array(c, dtype=np.float64, copy=True) for c in orb]
    skip = set(skip_solve_species or ())
    sources_for_target = {}
    for (tgt, src) in K_sources_per_bin[0].keys():
        sources_for_target.setdefault(tgt, []).append(src)
    order = [s for s in _SOLVE_ORDER if s < n_species] + [s for s in range(n_species) if s >= len(_SOLVE_ORDER)]
    waves = _build_solve_waves(sources_for_target, order, skip)
    fresh_cache = {}
    kdiag_cache = {}

    def log(msg):
        if verbose:
            print(msg, flush=True)

    def name(s):
        return _SPECIES_NAMES[s] if s < len(_SPECIES_NAMES) else s

    def orbit_dev(s, snap_dev, snap_host):
        if s in snap_dev:
            return snap_dev[s]
        if s in snap_host:
            return torch.as_tensor(np.stack(snap_host[s]), device="cuda")
        raise KeyError(f"orbits[{s}] missing for a target; seed orbits are needed for cyclic source DAGs")

    def kdiag(tgt, src):
        key = (tgt, src)
        if key not in kdiag_cache:
            kdiag_cache[key] = torch.as_tensor(
                np.stack([_diag_of(K_sources_per_bin[t][key], N) for t in range(N_BINS)]), device="cuda")
        return kdiag_cache[key]

    for wave in waves:
        snap_dev, snap_host = dict(dev_orbits), dict(host_orbits)
        todo = []  # (s, E (8, N) device, warm)
        for s in wave:
            if s in skip and cached_orbits is not None and s in cached_orbits:
                host_orbits[s] = [np.array(c, copy=True) for c in cached_orbits[s]]
                dev_orbits.pop(s, None)
                log(f"  [{name(s)}]\n    [cache] skipped factor + solve (operator+RHS unchanged)")
                continue
            e_host = np.stack([np.asarray(x, dtype=np.float64) for x in _emissions_for(emissions_SN, s, N)])
            if extra_rhs_per_bin_per_species is not None and s in extra_rhs_per_bin_per_species:
                e_host = e_host + np.stack([np.asarray(x, dtype=np.float64)
                                            for x in extra_rhs_per_bin_per_species[s]])
            E = torch.as_tensor(np.ascontiguousarray(e_host), device="cuda")
            srcs = []
            for src in sources_for_target.get(s, []):
                if src not in snap_dev and src not in snap_host:
                    raise KeyError(f"orbits[{src}] missing for target s={s}; seed orbits are needed "
                                   "for cyclic source DAGs")
                shift = 1 if (endbin_keys is not None and (s, src) in endbin_keys) else 0
                srcs.append((kdiag(s, src), orbit_dev(src, snap_dev, snap_host), shift))
            if srcs:
                device.source_coupling(E, srcs, out=E)
            if not bool((E != 0).any()):
                dev_orbits[s] = torch.zeros((N_BINS + 1, N), dtype=torch.float64, device="cuda")
                host_orbits.pop(s, None)
                log(f"  [{name(s)}]\n    [zero-source] skipped factor + solve (RHS identically zero)")
                continue
            warm = None if c_warm_SN is None else np.asarray(c_warm_SN[s * N:(s + 1) * N], dtype=np.float64)
            todo.append((s, E, warm))
        if not todo:
            continue
        # group: species with cached factors solve in their cached batch, the rest in a new one
        groups = {}
        new = []
        for item in todo:
            s = item[0]
            if lu_cache is not None and s in lu_cache:
                ent = lu_cache[s]
                groups.setdefault(id(ent.fb), (ent.fb, []))[1].append((item, ent.set_index))
            else:
                new.append(item)
        if new:
            t0 = time.time()
            fb = FactorBatch(sym, len(new), precision)
            Ts = []
            for (s, _, _) in new:
                for t in range(N_BINS):
                    Ts.append(torch.as_tensor(
                        _stencil(L_species_per_bin[t][s], sym), device="cuda"))
            fb.numeric(Ts, None, DTAU)
            torch.cuda.synchronize()
            log(f"  factored {len(new)} species x 8 bins on the device in {time.time() - t0:.2f}s")
            groups[id(fb)] = (fb, [(item, q) for q, item in enumerate(new)])
        for fb, members in groups.values():
            t1 = time.time()
            nm = len(members)
            slot_fb = fb
            if nm != fb.n_orbits or any(q != k for k, (_, q) in enumerate(members)):
                # solve slots 0..nm-1 mapped onto the members' factor sets
                slot_fb = _remap(fb, [q for (_, q) in members])
            E = torch.stack([it[1] for it, _ in members])
            warm = None
            if any(it[2] is not None for it, _ in members):
                warm = torch.as_tensor(np.stack([it[2] if it[2] is not None else np.zeros(N)
                                                 for it, _ in members]), device="cuda")
            orb, info = slot_fb.solve(E, c_warm=warm, tol=tol, maxiter=maxiter)
            for k, (it, q) in enumerate(members):
                s = it[0]
                dev_orbits[s] = orb[k]
                host_orbits.pop(s, None)
                gmres_iters[s] = int(info[k, 0])
                gmres_resid[s] = float(info[k, 1])
                periodicity[s] = float(info[k, 2])
                fresh_cache[s] = SpeciesFactors(fb, q)
                if verbose:
                    neg = int((orb[k] < 0).sum())
                    log(f"  [{name(s)}]\n"
                        f"    GMRES: {int(info[k, 0])} iter ({time.time() - t1:.2f}s batch of {nm}), "
                        f"resid={info[k, 1]:.1e}, period={info[k, 2]:.1e}, neg={neg}/{orb[k].numel()}")
                if keep_lu_species is not None and s not in keep_lu_species:
                    fresh_cache.pop(s, None)
                for t in range(N_BINS):
                    L_species_per_bin[t][s] = None
    orbits = dict(host_orbits)
    for s, o in dev_orbits.items():
        oh = o.cpu().numpy()
        orbits[s] = [oh[t].copy() for t in range(N_BINS + 1)]
    result = {"orbits": orbits, "gmres_iters": gmres_iters, "gmres_resid": gmres_resid,
              "periodicity": periodicity}
    if return_lu_cache:
        result["lu_cache"] = fresh_cache
    return result


def _stencil(L, sym):
    from .grid import stencil_from_matrix
    if L is None:
        raise ValueError("operator already released (solved earlier in this call)")
    return stencil_from_matrix(L, sym.nz, sym.ny, sym.nx, periodic=getattr(sym, "periodic", False))


class _SlotView:
    """A FactorBatch whose first solve slots are mapped onto chosen factor sets."""

    def __init__(self, fb, sets):
        self.fb = fb
        self.sets = sets

    def solve(self, E, **kw):
        m = list(self.sets) + [self.sets[-1]] * (self.fb.n_orbits - len(self.sets))
        self.fb.map(m)
        try:
            return self.fb.solve(E, **kw)
        finally:
            self.fb.map([o % self.fb.n_sets for o in range(self.fb.n_orbits)])


def _remap(fb, sets):
    return _SlotView(fb, sets)
