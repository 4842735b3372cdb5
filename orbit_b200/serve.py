"""Serving loop: continuous batching of periodic-orbit requests on one GPU.

Requests (forward, marginal or adjoint-receptor orbit solves of some species
on some domain and month) arrive at any time.  Factors are cached per
(domain, month): one factor set per species of that met month, resident in
HBM, reused by every later request for it.  Admission is by device memory:
a (domain, month) entry is created only when its factor storage and
workspace fit in the HBM budget, evicting idle least-recently-used entries
first; requests for entries that cannot be admitted wait.  Each worker
thread owns a CUDA stream; it takes the oldest waiting request whose entry is
idle, packs every waiting request of the same entry and direction into the
entry's solve slots (up to its capacity), maps each slot onto its species'
factor set and runs one batched GMRES.  Requests that arrive while a batch
runs join the next batch of their entry; batches of different entries run
concurrently on different streams.  Latency is measured from arrival to the
host-side completion of the request's batch.

This is the serving counterpart of the reference's per-species loops
(orbit/core/orbit.py:468-806, orbit/modes/adjoint.py) for a stream of
independent requests.
"""
from __future__ import annotations

import itertools
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import device
from .symbolic import Symbolic
from .synthetic import DTAU, N_BINS, MetBin

KINDS = ("forward", "marginal", "adjoint")


@dataclass
class OrbitRequest:
    domain: Tuple[int, int, int]
    month: int
    kind: str
    species: List[int]
    forcing: np.ndarray            # (len(species), 8, N): emissions, perturbations or receptors
    tol: float = 1e-6
    maxiter: int = 200
    id: int = -1
    t_arrive: float = 0.0
    t_start: float = 0.0
    t_done: float = 0.0
    result: Optional[np.ndarray] = None   # (len(species), 9, N)
    info: Optional[np.ndarray] = None
    error: Optional[str] = None
    done: threading.Event = field(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrive

    @property
    def direction(self) -> str:
        return "adjoint" if self.kind == "adjoint" else "forward"


class _Entry:
    """Factors of all species of one (domain, month), plus solve slots."""

    def __init__(self, key, sym, mets, sinks, slots, precision):
        self.key = key
        self.sym = sym
        self.mets_host = mets
        self.sinks_host = sinks          # list over species of (8, N)
        self.n_species = len(sinks)
        self.slots = slots
        self.precision = precision
        self.fb: Optional[device.FactorBatch] = None
        self.busy = False
        self.last_used = 0.0
        vb = 4 if precision == 32 else 8
        info = sym.info
        scratch = 2 * info["front_elems"] * vb + (info["tc_pack_floats"] * 4 if precision == 32 else 0)
        self.bytes = (self.n_species * N_BINS * (info["factor_elems"] * vb + 7 * sym.N * 8)
                      + min(48 << 30, self.n_species * N_BINS * scratch)
                      + slots * 60 * sym.N * 8)

    def build(self):
        """Assemble and factor every species of the entry (on the caller's stream)."""
        mets = [device.MetDevice(g) for g in self.mets_host]
        T = [device.assemble_transport(m) for m in mets]
        sinks = [torch.as_tensor(d[t], device="cuda") for d in self.sinks_host for t in range(N_BINS)]
        fb = device.FactorBatch(self.sym, self.slots, self.precision, n_sets=self.n_species)
        fb.numeric([T[t] for _ in range(self.n_species) for t in range(N_BINS)], sinks, DTAU)
        self.fb = fb

    def release(self):
        if self.fb is not None:
            self.fb.close()
            self.fb = None


class OrbitServer:
    """Continuous-batching request loop under an HBM budget.

    ``met_provider(domain, month) -> (mets, sinks)`` supplies the eight bins of
    meteorology (MetBin) and, per species, its (8, N) sink diagonal.
    """

    def __init__(self, met_provider: Callable, hbm_budget_bytes: float = 150e9, slots: int = 24,
                 precision: int = 32, workers: int = 2):
        self.met_provider = met_provider
        self.budget = float(hbm_budget_bytes)
        self.slots = int(slots)
        self.precision = int(precision)
        self.n_workers = int(workers)
        self._syms: Dict[tuple, Symbolic] = {}
        self._entries: Dict[tuple, _Entry] = {}
        self._pending: List[OrbitRequest] = []
        self._lock = threading.Condition()
        self._ids = itertools.count()
        self._stop = False
        self._threads: List[threading.Thread] = []
        self.completed: List[OrbitRequest] = []
        self.batches = 0
        self.orbits = 0

    # -- public ---------------------------------------------------------------
    def start(self):
        for w in range(self.n_workers):
            t = threading.Thread(target=self._worker, args=(w,), daemon=True)
            t.start()
            self._threads.append(t)
        return self

    def submit(self, req: OrbitRequest) -> OrbitRequest:
        if req.kind not in KINDS:
            raise ValueError(f"kind must be one of {KINDS}")
        req.id = next(self._ids)
        req.t_arrive = time.perf_counter()
        with self._lock:
            self._pending.append(req)
            self._lock.notify_all()
        return req

    def stop(self):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        for t in self._threads:
            t.join()
        for e in self._entries.values():
            e.release()

    def used_bytes(self) -> float:
        return sum(e.bytes for e in self._entries.values() if e.fb is not None or e.busy)

    # -- scheduling -------------------------------------------------------------
    def _sym(self, domain):
        if domain not in self._syms:
            self._syms[domain] = Symbolic(*domain)
        return self._syms[domain]

    def _admit(self, key) -> Optional[_Entry]:
        """Entry for key if it exists or fits the budget (evicting idle LRU entries)."""
        e = self._entries.get(key)
        if e is not None:
            return e
        domain, month = key
        mets, sinks = self.met_provider(domain, month)
        e = _Entry(key, self._sym(domain), mets, sinks, self.slots, self.precision)
        while self.used_bytes() + e.bytes > self.budget:
            idle = [x for x in self._entries.values() if not x.busy]
            if not idle:
                return None
            victim = min(idle, key=lambda x: x.last_used)
            victim.release()
            del self._entries[victim.key]
        self._entries[key] = e
        return e

    def _take_batch(self):
        """Oldest runnable request plus compatible waiting requests (lock held)."""
        for i, r in enumerate(self._pending):
            key = (tuple(r.domain), r.month)
            e = self._entries.get(key)
            if e is not None and e.busy:
                continue
            e = self._admit(key)
            if e is None:
                continue
            batch, used = [], 0
            for q in list(self._pending):
                if (tuple(q.domain), q.month) == key and q.direction == r.direction \
                        and used + len(q.species) <= e.slots:
                    batch.append(q)
                    used += len(q.species)
            if not batch:  # a single request larger than the slots: solve it alone in pieces
                batch = [r]
            for q in batch:
                self._pending.remove(q)
            e.busy = True
            return e, batch
        return None, None

    def _worker(self, w):
        stream = torch.cuda.Stream()
        while True:
            with self._lock:
                e, batch = None, None
                while not self._stop:
                    e, batch = self._take_batch()
                    if e is not None:
                        break
                    self._lock.wait(timeout=0.05)
                if e is None:
                    return
            try:
                with torch.cuda.stream(stream):
                    self._run(e, batch)
            except Exception as exc:  # report per request, keep serving
                for q in batch:
                    q.error = repr(exc)
                    q.t_done = time.perf_counter()
                    q.done.set()
            finally:
                with self._lock:
                    e.busy = False
                    e.last_used = time.perf_counter()
                    self._lock.notify_all()

    def _run(self, e: _Entry, batch: Sequence[OrbitRequest]):
        t0 = time.perf_counter()
        for q in batch:
            q.t_start = t0
        if e.fb is None:
            e.build()
        slots, forcing, tols, owners = [], [], [], []
        for q in batch:
            for k, s in enumerate(q.species):
                slots.append(s)
                forcing.append(q.forcing[k])
                owners.append((q, k))
            tols.append(q.tol)
        n = len(slots)
        for start in range(0, n, e.slots):
            part = slice(start, min(n, start + e.slots))
            sl = slots[part]
            e.fb.map(sl + [sl[-1]] * (e.slots - len(sl)))
            F = torch.as_tensor(np.stack(forcing[part]), device="cuda")
            tol = min(tols)
            maxiter = max(q.maxiter for q in batch)
            if batch[0].direction == "adjoint":
                out, info = e.fb.solve_adjoint(F, tol=tol, maxiter=maxiter)
            else:
                out, info = e.fb.solve(F, tol=tol, maxiter=maxiter)
            out = out.cpu().numpy()
            for j, (q, k) in enumerate(owners[part]):
                if q.result is None:
                    q.result = np.empty((len(q.species), N_BINS + 1, e.sym.N))
                    q.info = np.empty((len(q.species), 8))
                q.result[k] = out[j]
                q.info[k] = info[j]
        now = time.perf_counter()
        with self._lock:
            self.batches += 1
            self.orbits += n
        for q in batch:
            q.t_done = now
            self.completed.append(q)
            q.done.set()
