"""Device-side objects over the C ABI: met fields, transport stencils, factor
batches (chained solves, periodic-orbit GMRES), FCT source, mass balance.

Device memory is torch CUDA tensors (plumbing only); every computation runs
in liborbit_b200's sm_100a kernels on the tensor's stream.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .symbolic import Symbolic
from .synthetic import MetBin, DTAU, N_BINS

_MET_FIELDS = ("dP", "Dz", "u", "v", "u_plus", "u_minus", "v_plus", "v_minus", "u_e", "u_plus_e",
               "v_n", "v_plus_n", "kxxyy", "kzz", "w_plus", "w_minus", "cmfmc", "kmu", "kmv", "lat")


def _stream(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("orbit_b200 device path needs a CUDA device (no CPU fallback)")


class MetDevice:
    """One bin's meteorology resident on the device (fields as in MetBin)."""

    def __init__(self, met: MetBin, device="cuda"):
        _require_cuda()
        self.nz, self.ny, self.nx = met.nz, met.ny, met.nx
        self.N = met.N
        self.split = bool(met.split)
        self.dlat, self.dlon = float(met.dlat), float(met.dlon)
        self.t = {}
        for name in _MET_FIELDS:
            a = getattr(met, name)
            if name in ("kmu", "kmv") and met.split:
                continue
            if name == "cmfmc" and (a.size == 0 or not np.any(a)):
                continue
            self.t[name] = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device)
        self.pressure_form = not bool(getattr(met, "concentration_state", True))
        self.periodic = bool(getattr(met, "periodic_lon", False))
        if self.periodic:
            if self.nx < 3:
                raise ValueError("a periodic-longitude grid needs nx >= 3")
            for name in ("u_wrap", "u_plus_wrap", "u_minus_wrap", "kmu_wrap"):
                a = getattr(met, name, None)
                if a is None or (name == "kmu_wrap" and self.split):
                    continue
                self.t[name] = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64).reshape(self.nz, self.ny),
                                               device=device)
        # state weights: rho in the concentration form, 1 in the pressure form
        rho = met.state_weights().reshape(-1)
        self.rho = torch.as_tensor(rho, device=device)
        self.rebind()

    def rebind(self):
        """Rebuild the C struct from ``self.t`` (after its tensors were replaced,
        e.g. by views into one contiguous buffer that a single copy fills)."""
        self.struct = _lib.MetT(**{k: _lib.ptr(self.t.get(k)) for k in _MET_FIELDS},
                                dlat=self.dlat, dlon=self.dlon, split=int(self.split),
                                pressure_form=int(self.pressure_form), periodic_lon=int(self.periodic),
                                **{k: _lib.ptr(self.t.get(k))
                                   for k in ("u_wrap", "u_plus_wrap", "u_minus_wrap", "kmu_wrap")})


def assemble_transport(met: MetDevice, with_rowsum: bool = False):
    """K1: [7, N] transport stencil (concentration form unless the grid is in
    the pressure form) and, optionally, the pressure-form row sums."""
    T = torch.empty((7, met.N), dtype=torch.float64, device=met.rho.device)
    rs = torch.empty(met.N, dtype=torch.float64, device=met.rho.device) if with_rowsum else None
    _lib.check(_lib.lib().orbit_assemble_transport(met.nz, met.ny, met.nx, C.byref(met.struct),
                                                   _lib.ptr(T), _lib.ptr(rs), _stream()))
    return (T, rs) if with_rowsum else T


def boundary_loss(met: MetDevice) -> torch.Tensor:
    """Lateral boundary loss rate of every cell (N doubles, zero inside):
    the open-outflow part of the transport block's diagonal at the x (not
    on periodic grids) and y edges (operator.py:25-178)."""
    out = torch.empty(met.N, dtype=torch.float64, device=met.rho.device)
    _lib.check(_lib.lib().orbit_transport_boundary_loss(met.nz, met.ny, met.nx, C.byref(met.struct), _lib.ptr(out),
                                                        _stream()))
    return out


def stencil_to_csr(T: np.ndarray, nz: int, ny: int, nx: int, periodic: bool = False):
    """Host helper: scipy CSR of a [7, N] stencil (boundary entries dropped;
    with ``periodic`` the W entry of column 0 and the E entry of column nx-1
    are the wrap-face couplings to column nx-1 and column 0)."""
    import scipy.sparse as sp
    N = nz * ny * nx
    c = np.arange(N)
    k, r = np.divmod(c, nx * ny)
    j, i = np.divmod(r, nx)
    off = [np.zeros(N, np.int64), np.where(i > 0, -1, nx - 1), np.where(i < nx - 1, 1, -(nx - 1)),
           -nx, nx, -nx * ny, nx * ny]
    px = bool(periodic) and nx >= 3
    ok = [np.ones(N, bool), (i > 0) | px, (i < nx - 1) | px, j > 0, j < ny - 1, k > 0, k < nz - 1]
    rows, cols, vals = [], [], []
    for d in range(7):
        m = ok[d]
        o = off[d][m] if isinstance(off[d], np.ndarray) else off[d]
        rows.append(c[m]); cols.append(c[m] + o); vals.append(T[d][m])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(N, N))


SPECIES_FIELD_NAMES = ("Dz", "particle_dry_dep", "nh3_dry_dep", "so2_dry_dep", "nox_dry_dep", "hno3_dry_dep",
                       "o3_dry_dep", "is_land", "voc_dry_dep", "particle_wet_dep", "other_gas_wet_dep",
                       "so2_wet_dep", "nh_part", "no3_part", "fp_vbs", "fp_vbs_surface", "j_no2", "so2_ox",
                       "nox_ox", "o3_loss", "co_loss", "archive_oh")
N_SPECIES_ALL = 14
# (target, source) of the rows of the coupling output, in order
COUPLINGS = ((5, 3), (6, 4), (0, 12), (9, 0), (10, 9), (11, 10))


def species_diagonals(nz: int, ny: int, nx: int, fields: dict, a_photo: float = 0.0, k_age: float = 0.0,
                      aging_gain: float = 1.0, device="cuda"):
    """K1b: (14, N) species sink diagonals and (6, N) source-coupling diagonals
    of one bin from its per-cell fields (names as ``SPECIES_FIELD_NAMES``;
    optional fields may be missing or None)."""
    _require_cuda()
    N = nz * ny * nx
    keep = {}
    kw = {}
    for name in SPECIES_FIELD_NAMES:
        a = fields.get(name)
        if a is None:
            kw[name] = 0
            continue
        t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device) \
            if not isinstance(a, torch.Tensor) else a.to(device=device, dtype=torch.float64).contiguous()
        keep[name] = t
        kw[name] = _lib.ptr(t)
    st = _lib.SpeciesFieldsT(**kw, a_photo=float(a_photo), k_age=float(k_age), aging_gain=float(aging_gain))
    d = torch.empty((N_SPECIES_ALL, N), dtype=torch.float64, device=device)
    k = torch.empty((len(COUPLINGS), N), dtype=torch.float64, device=device)
    _lib.check(_lib.lib().orbit_species_diagonals(nz, ny, nx, C.byref(st), _lib.ptr(d), _lib.ptr(k), _stream()))
    return d, k


OXIDANT_FIELD_NAMES = ("temperature", "pressure", "oh", "no", "no2", "no3rad", "p_s", "p_nh", "p_no", "dust_fine",
                       "sea_salt_fine")


def nox_to_no3_rate(fields: dict, disable_night: bool = False, device="cuda") -> torch.Tensor:
    """Archive-driven NOx -> TotalNO3 rate (1/s) per cell from the oxidant
    fields (names as ``OXIDANT_FIELD_NAMES``; optional ones may be missing or None)."""
    _require_cuda()
    t = {}
    n = None
    for name in OXIDANT_FIELD_NAMES:
        a = fields.get(name)
        if a is None:
            continue
        t[name] = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64).reshape(-1), device=device)
        n = t[name].numel()
    if n is None:
        raise ValueError("no oxidant fields given")
    st = _lib.OxidantFieldsT(**{k: _lib.ptr(v) for k, v in t.items()})
    out = torch.empty(n, dtype=torch.float64, device=device)
    _lib.check(_lib.lib().orbit_nox_to_no3_rate(n, C.byref(st), int(bool(disable_night)), _lib.ptr(out), _stream()))
    return out


def source_coupling(e: torch.Tensor, sources, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """out[tau] = e[tau] - sum over sources of kdiag[tau] * c[tau + shift] for one
    target species; ``sources`` is a list of (kdiag (8, N), orbit (9, N), shift)."""
    e = e.contiguous()
    N = e.shape[-1]
    out = e.clone() if out is None else out
    if not sources:
        if out.data_ptr() != e.data_ptr():
            out.copy_(e)
        return out
    kd = torch.stack([s[0] for s in sources]).contiguous()
    orbs = [s[1].contiguous() for s in sources]
    cp = _lib.ptr_array([_lib.ptr(o) for o in orbs])
    sh = (C.c_int * len(sources))(*[int(s[2]) for s in sources])
    _lib.check(_lib.lib().orbit_source_coupling(N, len(sources), cp, sh, _lib.ptr(kd), _lib.ptr(e), _lib.ptr(out),
                                                _stream()))
    return out


def fct_source(met: MetDevice, c: torch.Tensor, dt: float = DTAU, limited: bool = True,
               c_ghost: Optional[torch.Tensor] = None):
    """K2: FCT deferred-correction source for one or more (N,) concentration
    vectors; ``c_ghost`` (same shape as ``c``) is the lateral-inflow field whose
    edge-cell values stand for the cells beyond the lateral edges."""
    c2 = c.reshape(-1, met.N).contiguous()
    d = torch.empty_like(c2)
    if c_ghost is None:
        _lib.check(_lib.lib().orbit_fct_source(met.nz, met.ny, met.nx, C.byref(met.struct), c2.shape[0],
                                               _lib.ptr(c2), float(dt), int(limited), _lib.ptr(d),
                                               _stream()))
    else:
        g2 = c_ghost.reshape(-1, met.N).contiguous()
        if g2.shape != c2.shape:
            raise ValueError("c_ghost must have the shape of c")
        _lib.check(_lib.lib().orbit_fct_source_ghost(met.nz, met.ny, met.nx, C.byref(met.struct), c2.shape[0],
                                                     _lib.ptr(c2), _lib.ptr(g2), float(dt), int(limited),
                                                     _lib.ptr(d), _stream()))
    return d.reshape(c.shape)


def fct_linear_operator(met: MetDevice, c_base: torch.Tensor, dt: float = DTAU) -> torch.Tensor:
    """Frozen-gain FCT operator L_AD of one or more baseline concentrations, as
    [7, N] stencils (vertical entries zero) in the transport blocks' layout."""
    c2 = c_base.reshape(-1, met.N).contiguous()
    out = torch.empty((c2.shape[0], 7, met.N), dtype=torch.float64, device=c2.device)
    _lib.check(_lib.lib().orbit_fct_linear_operator(met.nz, met.ny, met.nx, C.byref(met.struct), c2.shape[0],
                                                    _lib.ptr(c2), float(dt), _lib.ptr(out), _stream()))
    return out[0] if c_base.dim() == 1 else out


def stencil_apply(nz: int, ny: int, nx: int, stencils: torch.Tensor, x: torch.Tensor, alpha: float = 1.0,
                  trans: bool = False, out: Optional[torch.Tensor] = None, beta: float = 0.0,
                  periodic: bool = False) -> torch.Tensor:
    """out = beta out + alpha S x (or S^T x) for [.., 7, N] stencils and [.., N] vectors
    (``periodic``: the W/E entries of columns 0 and nx-1 are the wrap couplings)."""
    N = nz * ny * nx
    S2 = stencils.reshape(-1, 7, N).contiguous()
    x2 = x.reshape(-1, N).contiguous()
    if S2.shape[0] != x2.shape[0]:
        raise ValueError("one stencil per vector")
    y = out if out is not None else torch.empty_like(x2)
    _lib.check(_lib.lib().orbit_stencil_apply_grid(nz, ny, nx, int(bool(periodic)), x2.shape[0], _lib.ptr(S2),
                                                   _lib.ptr(x2), float(alpha), float(beta), int(trans), _lib.ptr(y),
                                                   _stream()))
    return y.reshape(x.shape)


def mass_balance(mets: Sequence[MetDevice], stencils: Sequence[torch.Tensor]) -> dict:
    """K7 row sums on the device, then the same order statistics the reference
    reports (operator.py:598-652): median, p90, p99, max of the interior rows
    and the top layer, per-layer p90."""
    g = mets[0]
    nz, ny, nx = g.nz, g.ny, g.nx
    nb = len(mets)
    dev = g.rho.device
    oi = torch.empty((nb, nz - 1, ny - 2, nx - 2), dtype=torch.float64, device=dev)
    ot = torch.empty((nb, ny - 2, nx - 2), dtype=torch.float64, device=dev)
    Tp = _lib.ptr_array([_lib.ptr(t) for t in stencils])
    Rp = _lib.ptr_array([_lib.ptr(m.rho) for m in mets])
    _lib.check(_lib.lib().orbit_mass_balance_rows(nz, ny, nx, nb, Tp, Rp, _lib.ptr(oi), _lib.ptr(ot),
                                                  _stream()))
    ri = oi.reshape(-1)
    rt = ot.reshape(-1)
    q = torch.tensor([0.5, 0.9, 0.99], dtype=torch.float64, device=dev)
    qi = torch.quantile(ri, q)
    qt = torch.quantile(rt, q[:2])
    per_layer = torch.cat([oi, ot[:, None]], dim=1)  # (nb, nz, ny-2, nx-2)
    lp90 = torch.stack([torch.quantile(per_layer[:, k].reshape(-1), 0.9) for k in range(nz)])
    return {
        "interior_median": float(qi[0]), "interior_p90": float(qi[1]), "interior_p99": float(qi[2]),
        "interior_max": float(ri.max()),
        "interior_frac_above_0.01": float((ri > 0.01).double().mean()),
        "interior_frac_above_0.1": float((ri > 0.1).double().mean()),
        "top_median": float(qt[0]), "top_p90": float(qt[1]),
        "layer_p90": [float(v) for v in lp90],
    }


class FactorBatch:
    """n_orbits x 8 numeric factorizations sharing a Symbolic, plus the chained
    solves and the periodic-orbit GMRES that run on them."""

    def __init__(self, sym: Symbolic, n_orbits: int, precision: int = 64,
                 n_sets: Optional[int] = None, n_bins: int = N_BINS):
        _require_cuda()
        self.sym = sym
        self.n_orbits = int(n_orbits)
        self.n_sets = int(n_sets) if n_sets is not None else self.n_orbits
        self.n_bins = int(n_bins)
        self.precision = int(precision)
        h = C.c_void_p()
        _lib.check(_lib.lib().orbit_factor_create_ex(sym.handle, self.n_orbits, self.n_sets, self.n_bins,
                                                     self.precision, C.byref(h)))
        self._h = h
        self.n_factored = 0
        self.N = sym.N

    def map(self, set_of_orbit: Sequence[int]):
        """Factor set of each solve slot (many right-hand sides may share one set)."""
        a = np.ascontiguousarray(np.asarray(set_of_orbit, dtype=np.int32))
        if a.shape != (self.n_orbits,):
            raise ValueError(f"need {self.n_orbits} set indices")
        _lib.check(_lib.lib().orbit_factor_map(self._h, a.ctypes.data))

    def numeric(self, T_stencils: Sequence[torch.Tensor], sinks: Optional[Sequence[torch.Tensor]],
                dtau: float = DTAU):
        """Factor len(T_stencils)//n_bins factor sets; lists are set-major, bin-minor."""
        n_inst = len(T_stencils)
        nb = self.n_bins
        if n_inst % nb or n_inst // nb > self.n_sets:
            raise ValueError(f"need {nb} stencils per factor set, at most {self.n_sets} sets")
        tp = _lib.ptr_array([_lib.ptr(t) for t in T_stencils])
        dp = _lib.ptr_array([_lib.ptr(d) for d in sinks]) if sinks is not None else None
        _lib.check(_lib.lib().orbit_factor_numeric(self._h, n_inst // nb, tp, dp, float(dtau),
                                                   _stream()))
        self.n_factored = n_inst // nb
        self.dtau = float(dtau)

    def chain(self, x: torch.Tensor, trans: bool = False, tau0: int = 0, tau1: int = N_BINS,
              forcing: Optional[torch.Tensor] = None, fscale: float = 1.0, refine: bool = True):
        """x: (n, N) -> P_{tau1-1}...P_{tau0} x (or the transposed chain)."""
        x = x.reshape(-1, self.N).contiguous()
        n = x.shape[0]
        out = torch.empty_like(x)
        if tau1 > self.n_bins:
            tau1 = self.n_bins
        f = forcing.reshape(n, N_BINS, self.N).contiguous() if forcing is not None else None
        _lib.check(_lib.lib().orbit_chain_apply(self._h, n, int(trans), int(tau0), int(tau1),
                                                _lib.ptr(x), _lib.ptr(out), _lib.ptr(f), float(fscale),
                                                int(refine), _stream()))
        return out

    def solve(self, e: torch.Tensor, c_warm: Optional[torch.Tensor] = None, tol: float = 1e-6,
              maxiter: int = 200, restart: int = 30, dtau: float = DTAU):
        """Periodic orbits of the first n orbits: e (n, 8, N) -> (orbit (n, 9, N), info (n, 8))."""
        e = e.reshape(-1, N_BINS, self.N).contiguous()
        n = e.shape[0]
        out = torch.empty((n, N_BINS + 1, self.N), dtype=torch.float64, device=e.device)
        info = np.zeros((n, 8))
        w = c_warm.reshape(n, self.N).contiguous() if c_warm is not None else None
        rc = _lib.lib().orbit_gmres_solve(self._h, n, _lib.ptr(e), float(dtau), _lib.ptr(w), float(tol),
                                          int(maxiter), int(restart), _lib.ptr(out), info.ctypes.data,
                                          _stream())
        if rc == 6:  # non-convergence: the reference warns and returns (orbit.py:184-186)
            print(f"    WARNING: GMRES did not converge for some orbits (iters={info[:, 0].tolist()})")
        else:
            _lib.check(rc)
        return out, info

    def solve_adjoint(self, R: torch.Tensor, lam_warm: Optional[torch.Tensor] = None,
                      tol: float = 1e-6, maxiter: int = 200, restart: int = 30):
        R = R.reshape(-1, N_BINS, self.N).contiguous()
        n = R.shape[0]
        out = torch.empty((n, N_BINS + 1, self.N), dtype=torch.float64, device=R.device)
        info = np.zeros((n, 8))
        w = lam_warm.reshape(n, self.N).contiguous() if lam_warm is not None else None
        rc = _lib.lib().orbit_adjoint_gmres_solve(self._h, n, _lib.ptr(R), _lib.ptr(w), float(tol),
                                                  int(maxiter), int(restart), _lib.ptr(out),
                                                  info.ctypes.data, _stream())
        if rc == 6:
            print(f"    WARNING: adjoint GMRES did not converge (iters={info[:, 0].tolist()})")
        else:
            _lib.check(rc)
        return out, info

    def profile(self, mode: int):
        """1: enable+reset, 0: disable+reset, 2: read -> dict of chain/factor timings."""
        out = (C.c_double * 6)()
        _lib.check(_lib.lib().orbit_factor_profile(self._h, int(mode), out))
        if mode != 2:
            return None
        return {"chain_launches": int(out[0]), "chain_ms": out[1], "chain_bytes": out[2],
                "factor_calls": int(out[3]), "factor_ms": out[4], "factor_flops": out[5]}

    def bytes(self):
        a, b = C.c_int64(), C.c_int64()
        _lib.check(_lib.lib().orbit_factor_bytes(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().orbit_factor_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_launches() -> int:
    """Kernels liborbit_b200 has launched so far (process-wide)."""
    return int(_lib.lib().orbit_kernel_launches())


INFO_FIELDS = ("gmres_iters", "residual", "periodicity", "neg_frac", "converged", "s_norm",
               "outer_refinements", "matvecs")


def info_dict(row) -> dict:
    d = {k: float(v) for k, v in zip(INFO_FIELDS, row)}
    d["gmres_iters"] = int(d["gmres_iters"])
    return d
