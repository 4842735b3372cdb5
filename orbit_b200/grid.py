"""Adapters between the reference's GridData and this package's MetBin.

``met_from_griddata`` reads any object with the reference ``GridData``
attributes (orbit/core/grid_data.py:19-215) and applies the reference's own
field conventions: the outer east/north faces follow ``edge_face``
(grid_data.py:558-576: the true face when the grid carries it, the edge
cell's face otherwise); the interface mass flux follows ``interface_omega``
(orbit/core/advection.py:383-411: ``omega_edge_plus/minus`` when present,
else the cell-centred split omega on interior interfaces with closed ground
and top; the ground is closed in every case); the non-split mode uses
max(+-U, 0) and adds the face meander diffusivity (convdiff.py:101-124).
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from .synthetic import MetBin


def _arr(g, name, default=None):
    a = getattr(g, name, None)
    if a is None:
        return default
    a = np.asarray(a, dtype=np.float64)
    return a if a.size else default


def met_from_griddata(g) -> MetBin:
    """MetBin view of a reference GridData (regional or periodic in longitude;
    the wrap face reads UAvg_wrap, UAvg_plus/minus_wrap and K_meander_u_wrap,
    grid_data.py:426-445)."""
    nz, ny, nx = int(g.nz), int(g.ny), int(g.nx)
    split = bool(getattr(g, "has_split_fluxes", False))
    u, v = _arr(g, "UAvg"), _arr(g, "VAvg")
    if split:
        up, um = _arr(g, "UAvg_plus"), _arr(g, "UAvg_minus")
        vp, vm = _arr(g, "VAvg_plus"), _arr(g, "VAvg_minus")
    else:
        up, um = np.maximum(u, 0.0), np.maximum(-u, 0.0)
        vp, vm = np.maximum(v, 0.0), np.maximum(-v, 0.0)

    def edge(true_name, proxy, axis_last):
        t = _arr(g, true_name)
        if t is not None:
            return t
        return proxy[:, :, -1] if axis_last else proxy[:, -1, :]

    u_e = edge("U_face_e", u, True)
    u_plus_e = edge("U_plus_face_e", _arr(g, "UAvg_plus", np.maximum(u, 0.0)), True)
    v_n = edge("V_face_n", v, False)
    v_plus_n = edge("V_plus_face_n", _arr(g, "VAvg_plus", np.maximum(v, 0.0)), False)
    wp_e, wm_e = _arr(g, "omega_edge_plus"), _arr(g, "omega_edge_minus")
    if wp_e is not None and wp_e.shape[0] == nz + 1:
        w_plus, w_minus = wp_e.copy(), wm_e.copy()
    else:
        w_plus = np.zeros((nz + 1, ny, nx))
        w_minus = np.zeros((nz + 1, ny, nx))
        op, om = _arr(g, "omega_plus"), _arr(g, "omega_minus")
        if op is not None:
            w_plus[1:nz] = op[1:]
            w_minus[1:nz] = om[1:]
    w_plus[0] = 0.0
    w_minus[0] = 0.0
    zeros = np.zeros((nz, ny, nx))
    cm = _arr(g, "CMFMC", np.zeros((nz + 1, ny, nx)))
    return MetBin(nz=nz, ny=ny, nx=nx, lat=np.asarray(g.lat, dtype=np.float64),
                  lon=np.asarray(getattr(g, "lon", np.zeros(nx)), dtype=np.float64),
                  dlat=float(g.dlat), dlon=float(g.dlon), dP=_arr(g, "dP"), Dz=_arr(g, "Dz"),
                  u=u, v=v, u_plus=up, u_minus=um, v_plus=vp, v_minus=vm, u_e=u_e,
                  u_plus_e=u_plus_e, u_minus_e=np.maximum(-u_e, 0.0), v_n=v_n, v_plus_n=v_plus_n,
                  v_minus_n=np.maximum(-v_n, 0.0), kxxyy=_arr(g, "Kxxyy"), kzz=_arr(g, "Kzz"),
                  w_plus=w_plus, w_minus=w_minus, cmfmc=cm,
                  kmu=_arr(g, "K_meander_u", zeros), kmv=_arr(g, "K_meander_v", zeros), split=split,
                  concentration_state=bool(getattr(g, "concentration_state", True)), **_wrap_fields(g, nx, split))


def _wrap_fields(g, nx, split):
    if not (bool(getattr(g, "periodic_lon", False)) and nx > 1):
        return {}
    if nx < 3:
        raise ValueError("a periodic-longitude grid needs nx >= 3 on the device path")
    uw = _arr(g, "UAvg_wrap")
    if uw is None:
        raise ValueError("periodic-longitude grid without UAvg_wrap")
    if split:
        upw, umw = _arr(g, "UAvg_plus_wrap"), _arr(g, "UAvg_minus_wrap")
    else:
        upw, umw = np.maximum(uw, 0.0), np.maximum(-uw, 0.0)
    return dict(periodic_lon=True, u_wrap=uw, u_plus_wrap=upw, u_minus_wrap=umw,
                kmu_wrap=_arr(g, "K_meander_u_wrap", np.zeros_like(uw)))


def griddata_like(m: MetBin, **extra) -> SimpleNamespace:
    """An object with the reference GridData attribute names for a MetBin."""
    w = m.w_plus - m.w_minus
    ns = SimpleNamespace(
        nz=m.nz, ny=m.ny, nx=m.nx, lat=m.lat, lon=m.lon, dlat=m.dlat, dlon=m.dlon, dP=m.dP, Dz=m.Dz,
        UAvg=m.u, VAvg=m.v, UAvg_plus=m.u_plus, UAvg_minus=m.u_minus, VAvg_plus=m.v_plus,
        VAvg_minus=m.v_minus, has_split_fluxes=m.split, U_face_e=m.u_e, U_plus_face_e=m.u_plus_e,
        U_minus_face_e=m.u_minus_e, V_face_n=m.v_n, V_plus_face_n=m.v_plus_n, V_minus_face_n=m.v_minus_n,
        Kzz=m.kzz, Kxxyy=m.kxxyy, K_meander_u=m.kmu, K_meander_v=m.kmv, omega_edge=w,
        omega_edge_plus=m.w_plus, omega_edge_minus=m.w_minus, has_interface_omega=True, CMFMC=m.cmfmc,
        periodic_lon=bool(m.periodic_lon), concentration_state=bool(m.concentration_state))
    if m.periodic_lon:
        ns.UAvg_wrap, ns.UAvg_plus_wrap, ns.UAvg_minus_wrap = m.u_wrap, m.u_plus_wrap, m.u_minus_wrap
        ns.K_meander_u_wrap = m.kmu_wrap if m.kmu_wrap is not None else np.zeros_like(m.u_wrap)
    for k, v in extra.items():
        setattr(ns, k, v)
    return ns


def stencil_from_matrix(M, nz: int, ny: int, nx: int, periodic: bool = False) -> np.ndarray:
    """[7, N] stencil of a sparse matrix on the 7-point pattern (raises if an
    entry lies outside it).  With ``periodic`` the wrap-face couplings of
    columns 0 and nx-1 go to their W and E entries."""
    import scipy.sparse as sp
    N = nz * ny * nx
    C = sp.csr_matrix(M)
    C.sum_duplicates()
    if C.shape != (N, N):
        raise ValueError(f"matrix shape {C.shape} does not match the grid ({N} cells)")
    rows = np.repeat(np.arange(N), np.diff(C.indptr))
    off = C.indices - rows
    st = np.zeros((7, N))
    k, r = np.divmod(rows, nx * ny)
    j, i = np.divmod(r, nx)
    offs = [(0, None), (-1, i > 0), (1, i < nx - 1), (-nx, j > 0), (nx, j < ny - 1),
            (-nx * ny, k > 0), (nx * ny, k < nz - 1)]
    used = np.zeros(len(rows), dtype=bool)
    for d, (o, ok) in enumerate(offs):
        m = off == o
        if ok is not None:
            m &= ok
        st[d, rows[m]] = C.data[m]
        used |= m
    if periodic and nx >= 3:
        for d, o, ok in ((1, nx - 1, i == 0), (2, -(nx - 1), i == nx - 1)):
            m = (off == o) & ok & ~used
            st[d, rows[m]] += C.data[m]
            used |= m
    if not np.all(used | (C.data == 0.0)):
        raise ValueError("matrix has entries outside the 7-point stencil of the grid")
    return st


def infer_grid_shape(M):
    """(nz, ny, nx) of a 7-point operator from its off-diagonal offsets
    (1, nx, nx*ny, and nx-1 for the wrap face of a periodic-longitude grid),
    or None when the pattern does not determine it."""
    import scipy.sparse as sp
    C = sp.csr_matrix(M)
    N = C.shape[0]
    rows = np.repeat(np.arange(N), np.diff(C.indptr))
    off = np.unique(np.abs(C.indices - rows))
    off = off[off > 0]
    if len(off) == 4 and off[0] == 1 and off[1] + 1 == off[2]:
        off = off[[0, 2, 3]]  # drop the wrap offset nx - 1
    if len(off) != 3 or off[0] != 1 or off[2] % off[1] or N % off[2]:
        return None
    nx, nxy = int(off[1]), int(off[2])
    return (N // nxy, nxy // nx, nx)


def infer_periodic(M, shape) -> bool:
    """True when the operator couples columns 0 and nx-1 of a row (the wrap
    face of a periodic-longitude grid, convdiff.py:150-202)."""
    import scipy.sparse as sp
    nz, ny, nx = shape
    if nx < 3:
        return False
    C = sp.csr_matrix(M)
    rows = np.repeat(np.arange(C.shape[0]), np.diff(C.indptr))
    off = C.indices - rows
    i = rows % nx
    return bool(np.any(((off == nx - 1) & (i == 0) | (off == -(nx - 1)) & (i == nx - 1)) & (C.data != 0.0)))
