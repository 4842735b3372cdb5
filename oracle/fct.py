"""Oracle: Zalesak-limited horizontal FCT deferred-correction source.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates:

* ``vanleer``                        orbit/core/fct.py:38-48
* ``_vanleer_phi``                   orbit/core/fct.py:235-247
* ``_horizontal_antidiffusive``      orbit/core/fct.py:256-357 (with or without ghost)
* ``_net_antidiffusive_into_cells``  orbit/core/fct.py:360-378
* ``_zalesak_2d``                    orbit/core/fct.py:381-447 (with or without ghost)
* ``compute_horizontal_fct_source``  orbit/core/fct.py:459-492
* ``assemble_fct_linear_operator``   orbit/core/fct.py:495-572
* the deferred-correction schedule   orbit/cli.py:1204-1241
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def vanleer(r):
    return (r + np.abs(r)) / (1.0 + np.abs(r))


def vanleer_phi(c_up, c_far, c_down):
    num = c_up - c_far
    den = c_down - c_up
    tiny = np.abs(den) < 1e-30
    r = num / np.where(tiny, 1e-30, den)
    r = np.where(tiny, np.where(np.abs(num) < 1e-30, 1.0, 1e6), r)
    return vanleer(r)


def _faces(g, c, ghost=None):
    """Anti-diffusive face fluxes and metric weights on x = c/rho; with a ghost
    field (x-space) its edge-cell values are the far-upwind values beyond the
    edges and the edge faces keep their reconstruction (fct.py:283-292)."""
    nz, ny, nx = g.nz, g.ny, g.nx
    out = {}
    split = g.split
    dx3 = np.broadcast_to(g.dx[None, :, None], (nz, ny, nx))
    if nx > 1:
        cL, cR = c[:, :, :-1], c[:, :, 1:]
        cLL = np.concatenate([cL[:, :, :1], c[:, :, :-2]], axis=2)
        cRR = np.concatenate([c[:, :, 2:], cR[:, :, -1:]], axis=2)
        if ghost is not None:
            cLL[:, :, 0] = ghost[:, :, 0]
            cRR[:, :, -1] = ghost[:, :, -1]
        pL = vanleer_phi(cL, cLL, cR)
        pR = vanleer_phi(cR, cRR, cL)
        if ghost is None:
            pL[:, :, 0] = 0.0
            pR[:, :, -1] = 0.0
        up = g.u_plus[:, :, 1:] if split else np.maximum(g.u[:, :, 1:], 0.0)
        um = g.u_minus[:, :, 1:] if split else np.maximum(-g.u[:, :, 1:], 0.0)
        beta = 0.5 * (up * pL + um * pR)
        A = beta * (cR - cL)
        d = dx3[:, :, 1:]
        dl, dr = g.dP[:, :, :-1], g.dP[:, :, 1:]
        face = 0.5 * (dl + dr)
        ok = (dl > 0) & (dr > 0)
        out["x"] = dict(A=A, beta=beta,
                        trL=np.where(ok, face / np.where(dl > 0, dl, 1.0), 1.0),
                        trR=np.where(ok, face / np.where(dr > 0, dr, 1.0), 1.0),
                        inv=1.0 / np.where(d > 0, d, 1.0), ok=ok)
    if ny > 1:
        cS, cN = c[:, :-1, :], c[:, 1:, :]
        cSS = np.concatenate([cS[:, :1, :], c[:, :-2, :]], axis=1)
        cNN = np.concatenate([c[:, 2:, :], cN[:, -1:, :]], axis=1)
        if ghost is not None:
            cSS[:, 0, :] = ghost[:, 0, :]
            cNN[:, -1, :] = ghost[:, -1, :]
        pS = vanleer_phi(cS, cSS, cN)
        pN = vanleer_phi(cN, cNN, cS)
        if ghost is None:
            pS[:, 0, :] = 0.0
            pN[:, -1, :] = 0.0
        vp = g.v_plus[:, 1:, :] if split else np.maximum(g.v[:, 1:, :], 0.0)
        vm = g.v_minus[:, 1:, :] if split else np.maximum(-g.v[:, 1:, :], 0.0)
        beta = 0.5 * (vp * pS + vm * pN)
        A = beta * (cN - cS)
        dxs, dxn = dx3[:, :-1, :], dx3[:, 1:, :]
        dxf = 0.5 * (dxs + dxn)
        ds, dn = g.dP[:, :-1, :], g.dP[:, 1:, :]
        face = 0.5 * (ds + dn)
        ok = (ds > 0) & (dn > 0)
        out["y"] = dict(A=A, beta=beta,
                        trL=np.where(ok, (dxf / dxs) * (face / np.where(ds > 0, ds, 1.0)), 1.0),
                        trR=np.where(ok, (dxf / dxn) * (face / np.where(dn > 0, dn, 1.0)), 1.0),
                        inv=1.0 / g.dy, ok=ok)
    return out


def _net(g, faces, Cx=None, Cy=None):
    d = np.zeros((g.nz, g.ny, g.nx))
    if "x" in faces:
        f = faces["x"]
        fl = (1.0 if Cx is None else Cx) * f["A"] * f["inv"]
        d[:, :, 1:] += np.where(f["ok"], f["trR"] * fl, 0.0)
        d[:, :, :-1] -= np.where(f["ok"], f["trL"] * fl, 0.0)
    if "y" in faces:
        f = faces["y"]
        fl = (1.0 if Cy is None else Cy) * f["A"] * f["inv"]
        d[:, 1:, :] += np.where(f["ok"], f["trR"] * fl, 0.0)
        d[:, :-1, :] -= np.where(f["ok"], f["trL"] * fl, 0.0)
    return d


def _zalesak(g, c, faces, dt, ghost=None):
    nz, ny, nx = g.nz, g.ny, g.nx
    o = c if ghost is None else ghost  # beyond an edge: ghost or clamped
    w = np.concatenate([o[:, :, :1], c[:, :, :-1]], axis=2)
    e = np.concatenate([c[:, :, 1:], o[:, :, -1:]], axis=2)
    s = np.concatenate([o[:, :1, :], c[:, :-1, :]], axis=1)
    n = np.concatenate([c[:, 1:, :], o[:, -1:, :]], axis=1)
    stk = np.stack([c, w, e, s, n])
    cmax, cmin = stk.max(0), stk.min(0)
    Pp = np.zeros((nz, ny, nx))
    Pm = np.zeros((nz, ny, nx))

    def into(key):
        f = faces[key]
        fl = f["A"] * f["inv"]
        return (np.where(f["ok"], f["trR"] * fl, 0.0), np.where(f["ok"], -f["trL"] * fl, 0.0))

    if "x" in faces:
        hi, lo = into("x")
        Pp[:, :, 1:] += np.maximum(hi, 0.0)
        Pm[:, :, 1:] += np.maximum(-hi, 0.0)
        Pp[:, :, :-1] += np.maximum(lo, 0.0)
        Pm[:, :, :-1] += np.maximum(-lo, 0.0)
    if "y" in faces:
        hi, lo = into("y")
        Pp[:, 1:, :] += np.maximum(hi, 0.0)
        Pm[:, 1:, :] += np.maximum(-hi, 0.0)
        Pp[:, :-1, :] += np.maximum(lo, 0.0)
        Pm[:, :-1, :] += np.maximum(-lo, 0.0)
    Qp = (cmax - c) / dt
    Qm = (c - cmin) / dt
    Rp = np.where(Pp > 0, np.minimum(1.0, Qp / np.where(Pp > 0, Pp, 1.0)), 0.0)
    Rm = np.where(Pm > 0, np.minimum(1.0, Qm / np.where(Pm > 0, Pm, 1.0)), 0.0)
    Cx = Cy = None
    if "x" in faces:
        hi, _ = into("x")
        Cx = np.clip(np.where(hi >= 0.0, np.minimum(Rp[:, :, 1:], Rm[:, :, :-1]),
                              np.minimum(Rm[:, :, 1:], Rp[:, :, :-1])), 0.0, 1.0)
    if "y" in faces:
        hi, _ = into("y")
        Cy = np.clip(np.where(hi >= 0.0, np.minimum(Rp[:, 1:, :], Rm[:, :-1, :]),
                              np.minimum(Rm[:, 1:, :], Rp[:, :-1, :])), 0.0, 1.0)
    return Cx, Cy


def fct_source(g, c_flat, dt, limited=True, c_ghost_flat=None):
    """d_AD = rho * (-div(C (.) A)) on x = c/rho (fct.py:459-492); rho is the
    state weight, 1 in the pressure form (_state_weights, fct.py:451-456);
    ``c_ghost_flat`` the lateral inflow field (fct.py:476-487)."""
    rho = g.state_weights().reshape(-1)
    c = (np.asarray(c_flat, dtype=np.float64) / rho).reshape(g.nz, g.ny, g.nx)
    ghost = None
    if c_ghost_flat is not None:
        ghost = (np.asarray(c_ghost_flat, dtype=np.float64) / rho).reshape(g.nz, g.ny, g.nx)
    faces = _faces(g, c, ghost)
    Cx, Cy = _zalesak(g, c, faces, dt, ghost) if limited else (None, None)
    return _net(g, faces, Cx, Cy).reshape(-1) * rho


def fct_linear_operator(g, c_base_flat, dt):
    """Frozen-gain 5-point L_AD with L_AD c_base = -d_AD(c_base) (fct.py:495-572)."""
    nz, ny, nx = g.nz, g.ny, g.nx
    N = nz * ny * nx
    rho = g.state_weights().reshape(-1)
    c = (np.asarray(c_base_flat, dtype=np.float64) / rho).reshape(nz, ny, nx)
    idx = np.arange(N).reshape(nz, ny, nx)
    faces = _faces(g, c)
    Cx, Cy = _zalesak(g, c, faces, dt)
    r, cc, v = [], [], []
    for key, C, lo, hi in (("x", Cx, idx[:, :, :-1], idx[:, :, 1:]),
                           ("y", Cy, idx[:, :-1, :], idx[:, 1:, :])):
        if key not in faces:
            continue
        f = faces[key]
        w = np.where(f["ok"], C * f["beta"] * f["inv"], 0.0)
        wR, wL = f["trR"] * w, f["trL"] * w
        for rr, col, val in ((hi, hi, -wR), (hi, lo, wR), (lo, hi, wL), (lo, lo, -wL)):
            r.append(rr.ravel()); cc.append(col.ravel()); v.append(val.ravel())
    L = sp.csc_matrix((np.concatenate(v), (np.concatenate(r), np.concatenate(cc))), shape=(N, N))
    return (sp.diags(rho) @ L @ sp.diags(1.0 / rho)).tocsc()
