"""Seeded synthetic meteorology and species fields for the periodic-orbit path.

The real ORBIT inputs (preprocessed MERRA-2 / WRF bin files on the South-Asia
grid) are not distributed with the reference, so every workload here is drawn
from fixed seeds with the shapes and value distributions of the reference's
benchmark configurations:

* horizontal grid 0.625 deg x 0.5 deg (``orbit/core/grid_data.py:35-36``),
  latitude origin 5 N, longitude origin 60 E;
* hybrid levels ``Ap = 6500 eta``, ``Bp = 1 - eta``; ``Psurf = 101325 Pa``
  (optionally perturbed by terrain, used by the parity tests only);
* ``Dz = dP / (rho_k g)`` with ``rho_k = 1.2`` (optionally a height profile);
* winds ``u, v ~ N(0, 8 m/s)`` drawn on the staggered faces, Gaussian-smoothed
  over 3 cells and rescaled back to an 8 m/s standard deviation; the cell
  value is the west/south face and the east/north outer faces are kept, as
  ``load_grid`` does (``grid_data.py:400-415``);
* the interface mass flux is diagnosed from the horizontal block's row sums
  by the rule ``w[k+1] = w[k] + R_h[k] dP_k`` with a closed ground
  (``tests/test_interface_omega_transport.py:139-143``);
* ``K_zz`` log-uniform on [0.1, 100] m^2/s, ``K_xxyy = 1e3`` m^2/s, no meander;
* optional convective mass flux (lognormal in 30 % of columns);
* per species: surface dry-deposition velocity U(0.001, 0.02) m/s, a
  first-order loss U(1e-6, 1e-4) 1/s and lognormal(0, 1.5) surface emissions
  scaled to 1e-9 ug m^-3 s^-1.

Nothing here is on the device hot path; it only produces inputs.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

EARTH_RADIUS = 6378137.0
GRAVITY = 9.80665
DEG_TO_RAD = np.pi / 180.0
N_BINS = 8
DTAU = 10800.0


@dataclass
class MetBin:
    """Averaged meteorology of one diurnal bin on an (nz, ny, nx) grid.

    Field meaning follows ``GridData`` (``orbit/core/grid_data.py:19-215``):
    ``u``/``v`` are the net west/south-face winds (UAvg/VAvg), ``u_plus``/
    ``u_minus`` and ``v_plus``/``v_minus`` the split-flux averages, ``*_e`` /
    ``*_n`` the true east/north outer faces, ``w_plus``/``w_minus`` the
    interface mass flux (Pa/s, index 0 = ground), ``cmfmc`` the convective
    updraft mass flux (kg/m^2/s, interface levels), ``kmu``/``kmv`` the
    face-centred meander diffusivity (used only when ``split`` is False).
    """
    nz: int
    ny: int
    nx: int
    lat: np.ndarray
    lon: np.ndarray
    dlat: float
    dlon: float
    dP: np.ndarray
    Dz: np.ndarray
    u: np.ndarray
    v: np.ndarray
    u_plus: np.ndarray
    u_minus: np.ndarray
    v_plus: np.ndarray
    v_minus: np.ndarray
    u_e: np.ndarray
    u_plus_e: np.ndarray
    u_minus_e: np.ndarray
    v_n: np.ndarray
    v_plus_n: np.ndarray
    v_minus_n: np.ndarray
    kxxyy: np.ndarray
    kzz: np.ndarray
    w_plus: np.ndarray
    w_minus: np.ndarray
    cmfmc: np.ndarray
    kmu: np.ndarray
    kmv: np.ndarray
    split: bool = True
    concentration_state: bool = True  # GridData.concentration_state (grid_data.py:71)
    # periodic longitude (GridData.periodic_lon, grid_data.py:426-445): the
    # wrap face between columns nx-1 and 0, (nz, ny) each
    periodic_lon: bool = False
    u_wrap: Optional[np.ndarray] = None
    u_plus_wrap: Optional[np.ndarray] = None
    u_minus_wrap: Optional[np.ndarray] = None
    kmu_wrap: Optional[np.ndarray] = None

    @property
    def N(self) -> int:
        return self.nz * self.ny * self.nx

    @property
    def dx(self) -> np.ndarray:
        return EARTH_RADIUS * np.cos(self.lat * DEG_TO_RAD) * self.dlon * DEG_TO_RAD

    @property
    def dy(self) -> float:
        return EARTH_RADIUS * self.dlat * DEG_TO_RAD

    def rho(self) -> np.ndarray:
        """dP / (g Dz), 1 where a cell is degenerate (``grid_data.py:543-554``)."""
        ok = (self.dP > 0) & (self.Dz > 0)
        return np.where(ok, self.dP / (GRAVITY * np.where(ok, self.Dz, 1.0)), 1.0)

    def state_weights(self) -> np.ndarray:
        """Weights of the transported state: rho in the concentration form, 1 in
        the pressure form (``_state_weights``, ``orbit/core/fct.py:451-456``;
        ``mass_balance_diagnostics``, ``orbit/core/operator.py:626``)."""
        if self.concentration_state:
            return self.rho()
        return np.ones((self.nz, self.ny, self.nx))


@dataclass
class SpeciesFields:
    """Per-species sinks and emissions (one species, all bins).

    ``vd`` (8, ny, nx) surface dry-deposition velocity (m/s), ``wet`` (8, nz,
    ny, nx) wet-deposition rate (1/s), ``loss`` (8, nz, ny, nx) first-order
    chemical loss (1/s), ``emis`` (8, N) emission rate in k-major cell order.
    The operator diagonal they add is ``wet + loss + [k=0] vd / Dz_0``, the
    structure of ``assemble_deposition`` plus the diagonal chemistry terms of
    ``assemble_species_operators`` (``orbit/core/deposition.py:101-146``,
    ``orbit/core/operator.py:555-585``).
    """
    vd: np.ndarray
    wet: np.ndarray
    loss: np.ndarray
    emis: np.ndarray

    def sink_diag(self, met: List[MetBin]) -> np.ndarray:
        """(8, N) diagonal sink rate of this species per bin."""
        out = []
        for tau, g in enumerate(met):
            d = self.wet[tau] + self.loss[tau]
            dz0 = g.Dz[0]
            d = d.copy()
            d[0] = d[0] + np.where(dz0 > 0, self.vd[tau] / np.where(dz0 > 0, dz0, 1.0), 0.0)
            out.append(d.reshape(-1))
        return np.stack(out)


def _smooth(field: np.ndarray, sigma: float, axes=(1, 2)) -> np.ndarray:
    from scipy.ndimage import gaussian_filter
    sig = [0.0] * field.ndim
    for a in axes:
        sig[a] = sigma
    return gaussian_filter(field, sigma=sig, mode="nearest")


def _wind(rng, nz, ny, nx, stag_axis, std=8.0, sigma=3.0):
    shape = [nz, ny, nx]
    shape[stag_axis] += 1
    f = rng.normal(0.0, std, size=shape)
    f = _smooth(f, sigma)
    sd = f.std()
    if sd > 0:
        f = f * (std / sd)
    return f


def horizontal_row_sums(g: MetBin) -> np.ndarray:
    """Row sums (1/s) of the pressure-form horizontal convection-diffusion block.

    Only used to diagnose a mass-consistent interface flux for synthetic
    inputs; diffusion cancels and the advective divergence remains.
    """
    nz, ny, nx = g.nz, g.ny, g.nx
    r = np.zeros((nz, ny, nx))
    dx = np.broadcast_to(g.dx[None, :, None], (nz, ny, nx))
    dP = g.dP
    if nx > 1:
        up, um = g.u_plus[:, :, 1:], g.u_minus[:, :, 1:]
        d = dx[:, :, 1:]
        pl, pr = dP[:, :, :-1], dP[:, :, 1:]
        face = 0.5 * (pl + pr)
        ok = (pl > 0) & (pr > 0)
        trr = np.where(ok, face / np.where(pr > 0, pr, 1.0), 1.0)
        trl = np.where(ok, face / np.where(pl > 0, pl, 1.0), 1.0)
        r[:, :, 1:] += trr * (um - up) / d
        r[:, :, :-1] += trl * (up - um) / d
    if g.periodic_lon:
        # wrap face: column nx-1 on its low side, column 0 on its high side
        up, um = g.u_plus_wrap, g.u_minus_wrap
        d = dx[:, :, 0]
        pl, pr = dP[:, :, -1], dP[:, :, 0]
        face = 0.5 * (pl + pr)
        ok = (pl > 0) & (pr > 0)
        trr = np.where(ok, face / np.where(pr > 0, pr, 1.0), 1.0)
        trl = np.where(ok, face / np.where(pl > 0, pl, 1.0), 1.0)
        r[:, :, 0] += trr * (um - up) / d
        r[:, :, -1] += trl * (up - um) / d
    else:
        r[:, :, 0] += np.where(g.u_minus[:, :, 0] > 0, g.u_minus[:, :, 0], 0.0) / dx[:, :, 0]
        r[:, :, -1] += np.where(g.u_plus_e > 0, g.u_plus_e, 0.0) / dx[:, :, -1]
    dy = g.dy
    dxc = g.dx
    if ny > 1:
        vp, vm = g.v_plus[:, 1:, :], g.v_minus[:, 1:, :]
        ps, pn = dP[:, :-1, :], dP[:, 1:, :]
        face = 0.5 * (ps + pn)
        dxs, dxn = dx[:, :-1, :], dx[:, 1:, :]
        dxf = 0.5 * (dxs + dxn)
        ok = (ps > 0) & (pn > 0)
        trn = np.where(ok, (dxf / dxn) * (face / np.where(pn > 0, pn, 1.0)), 1.0)
        trs = np.where(ok, (dxf / dxs) * (face / np.where(ps > 0, ps, 1.0)), 1.0)
        r[:, 1:, :] += trn * (vm - vp) / dy
        r[:, :-1, :] += trs * (vp - vm) / dy
    lat_s = g.lat[0] - g.dlat / 2.0
    lat_n = g.lat[-1] + g.dlat / 2.0
    tr_s = EARTH_RADIUS * np.cos(lat_s * DEG_TO_RAD) * g.dlon * DEG_TO_RAD / dxc[0]
    tr_n = EARTH_RADIUS * np.cos(lat_n * DEG_TO_RAD) * g.dlon * DEG_TO_RAD / dxc[-1]
    r[:, 0, :] += np.where(g.v_minus[:, 0, :] > 0, g.v_minus[:, 0, :], 0.0) / dy * tr_s
    r[:, -1, :] += np.where(g.v_plus_n > 0, g.v_plus_n, 0.0) / dy * tr_n
    return r


def make_met_bin(rng, nz, ny, nx, *, terrain_amp=0.0, rho_profile=False,
                 cmfmc_frac=0.0, lat0=5.0, lon0=60.0, dlat=0.5, dlon=0.625,
                 wind_std=8.0, split=True, periodic=False) -> MetBin:
    """Draw one bin of synthetic meteorology.  With ``periodic`` the grid wraps
    in longitude (dlon = 360 / nx) and the wrap face takes the mean of the
    first and last staggered winds, as the reference's loader does
    (grid_data.py:426-445)."""
    if periodic:
        if nx < 3:
            raise ValueError("a periodic-longitude grid needs nx >= 3")
        dlon = 360.0 / nx
    lat = lat0 + dlat * np.arange(ny)
    lon = lon0 + dlon * np.arange(nx)
    eta = np.linspace(0.0, 1.0, nz + 1)
    Ap = 6500.0 * eta
    Bp = 1.0 - eta
    Ps = np.full((ny, nx), 101325.0)
    if terrain_amp > 0:
        Ps = Ps - terrain_amp * _smooth(rng.random((1, ny, nx)), 2.0)[0] / 0.5
    P = Ap[:, None, None] + Bp[:, None, None] * Ps[None]
    dP = P[:-1] - P[1:]
    if rho_profile:
        zmid = np.cumsum(np.full(nz, 600.0)) - 300.0
        rho_k = 1.2 * np.exp(-zmid / 8000.0)
        rho3 = rho_k[:, None, None] * (1.0 + 0.05 * rng.random((nz, ny, nx)))
    else:
        rho3 = np.full((nz, ny, nx), 1.2)
    Dz = dP / (rho3 * GRAVITY)

    U = _wind(rng, nz, ny, nx, 2, std=wind_std)
    V = _wind(rng, nz, ny, nx, 1, std=wind_std)
    u, u_e = U[:, :, :nx].copy(), U[:, :, nx].copy()
    v, v_n = V[:, :ny, :].copy(), V[:, ny, :].copy()
    kzz = 10.0 ** rng.uniform(-1.0, 2.0, size=(nz, ny, nx))
    kxxyy = np.full((nz, ny, nx), 1.0e3)
    cmfmc = np.zeros((nz + 1, ny, nx))
    if cmfmc_frac > 0:
        active = rng.random((ny, nx)) < cmfmc_frac
        amp = np.exp(rng.normal(np.log(0.01), 1.0, size=(ny, nx))) * active
        prof = np.sin(np.pi * np.arange(nz + 1) / nz)
        cmfmc = prof[:, None, None] * amp[None]
        cmfmc[0] = 0.0
        cmfmc[nz] = 0.0
    zeros3 = np.zeros((nz, ny, nx))
    g = MetBin(nz=nz, ny=ny, nx=nx, lat=lat, lon=lon, dlat=dlat, dlon=dlon,
               dP=dP, Dz=Dz, u=u, v=v,
               u_plus=np.maximum(u, 0.0), u_minus=np.maximum(-u, 0.0),
               v_plus=np.maximum(v, 0.0), v_minus=np.maximum(-v, 0.0),
               u_e=u_e, u_plus_e=np.maximum(u_e, 0.0), u_minus_e=np.maximum(-u_e, 0.0),
               v_n=v_n, v_plus_n=np.maximum(v_n, 0.0), v_minus_n=np.maximum(-v_n, 0.0),
               kxxyy=kxxyy, kzz=kzz,
               w_plus=np.zeros((nz + 1, ny, nx)), w_minus=np.zeros((nz + 1, ny, nx)),
               cmfmc=cmfmc, kmu=zeros3.copy(), kmv=zeros3.copy(), split=split)
    if periodic:
        uw = 0.5 * (U[:, :, 0] + U[:, :, nx])
        g.periodic_lon = True
        g.u_wrap = uw
        g.u_plus_wrap = np.maximum(uw, 0.0)
        g.u_minus_wrap = np.maximum(-uw, 0.0)
        g.kmu_wrap = np.zeros((nz, ny))
    rh = horizontal_row_sums(g)
    w = np.zeros((nz + 1, ny, nx))
    w[1:] = np.cumsum(rh * dP, axis=0)
    g.w_plus = np.maximum(w, 0.0)
    g.w_minus = np.maximum(-w, 0.0)
    return g


def make_met(seed: int, nz: int, ny: int, nx: int, **kw) -> List[MetBin]:
    """Eight bins of meteorology from one seed (bins draw in sequence)."""
    rng = np.random.default_rng(seed)
    return [make_met_bin(rng, nz, ny, nx, **kw) for _ in range(N_BINS)]


def make_species(seed: int, nz: int, ny: int, nx: int, *, emis_scale=1e-9,
                 vd_range=(0.001, 0.02), loss_range=(1e-6, 1e-4),
                 wet=0.0) -> SpeciesFields:
    """Sinks and emissions of one species (seeded; identical emissions per bin)."""
    rng = np.random.default_rng(seed)
    N = nz * ny * nx
    vd1 = rng.uniform(*vd_range, size=(ny, nx))
    loss1 = rng.uniform(*loss_range, size=(nz, ny, nx))
    e = np.zeros((nz, ny, nx))
    e[0] = emis_scale * rng.lognormal(0.0, 1.5, size=(ny, nx))
    vd = np.broadcast_to(vd1, (N_BINS, ny, nx)).copy()
    loss = np.broadcast_to(loss1, (N_BINS, nz, ny, nx)).copy()
    wetf = np.full((N_BINS, nz, ny, nx), float(wet))
    emis = np.broadcast_to(e.reshape(-1), (N_BINS, N)).copy()
    return SpeciesFields(vd=vd, wet=wetf, loss=loss, emis=emis)


@dataclass
class Workload:
    """A named benchmark workload: met draws and species of one domain."""
    name: str
    nz: int
    ny: int
    nx: int
    met: List[List[MetBin]] = field(default_factory=list)
    species: List[SpeciesFields] = field(default_factory=list)
    tol: float = 1e-8
    seeds: dict = field(default_factory=dict)


def config_workload(config: int, n_species: Optional[int] = None,
                    n_met: Optional[int] = None, seed: int = 2024) -> Workload:
    """Synthetic stand-ins for the five benchmark configurations.

    0: 24x20x15, one species, tol 1e-10, no convection.
    1: 80x72x15, 12 species, convection in 30 % of columns, tol 1e-8.
    2: config 1 with 12 met draws (144 orbits), tol 1e-6 (mixed precision).
    3: config 1 operator, forward/adjoint right-hand sides, tol 1e-6.
    """
    if config == 0:
        nz, ny, nx, ns, nm, cf, tol = 15, 20, 24, 1, 1, 0.0, 1e-10
    elif config == 1:
        nz, ny, nx, ns, nm, cf, tol = 15, 72, 80, 12, 1, 0.3, 1e-8
    elif config == 2:
        nz, ny, nx, ns, nm, cf, tol = 15, 72, 80, 12, 12, 0.3, 1e-6
    elif config == 3:
        nz, ny, nx, ns, nm, cf, tol = 15, 72, 80, 1, 1, 0.3, 1e-6
    else:
        raise ValueError(f"unknown config {config}")
    if n_species is not None:
        ns = n_species
    if n_met is not None:
        nm = n_met
    wl = Workload(name=f"config{config}", nz=nz, ny=ny, nx=nx, tol=tol,
                  seeds={"met": [seed + 1000 * m for m in range(nm)],
                         "species": [seed + 17 + s for s in range(ns)]})
    for m in range(nm):
        wl.met.append(make_met(seed + 1000 * m, nz, ny, nx, cmfmc_frac=cf))
    for s in range(ns):
        wl.species.append(make_species(seed + 17 + s, nz, ny, nx))
    return wl
