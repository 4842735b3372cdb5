"""Oracle: transport-block and species-operator assembly (numpy/scipy).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates:

* ``_patankar_A``                         orbit/core/convdiff.py:16-39
* ``assemble_horizontal_convdiff``        orbit/core/convdiff.py:42-387
  (split and non-split flux modes; the periodic-longitude wrap face,
  convdiff.py:150-202)
* ``compute_lateral_boundary_loss``       orbit/core/operator.py:25-178
* ``interface_omega`` +
  ``assemble_vertical_advection``         orbit/core/advection.py:383-523
* ``assemble_vertical_diffusion``         orbit/core/mixing.py:14-117
* ``assemble_cmfmc_transport``            orbit/core/convection.py:25-140
* ``assemble_transport_block`` +
  ``to_concentration_form``               orbit/core/operator.py:281-353
* species operator ``L_s = T + diag(d_s)`` orbit/core/operator.py:371-595
* ``mass_balance_diagnostics``            orbit/core/operator.py:598-652

Inputs are ``orbit_b200.synthetic.MetBin`` objects (same field meaning as the
reference ``GridData``).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

EARTH_RADIUS = 6378137.0
GRAVITY = 9.80665
DEG_TO_RAD = np.pi / 180.0


def patankar_A(pe_abs):
    """A(|Pe|) = |Pe|/expm1(|Pe|) with the small/large guards (convdiff.py:16-39)."""
    pe_abs = np.asarray(pe_abs, dtype=np.float64)
    out = np.empty_like(pe_abs)
    lo = pe_abs < 1e-6
    hi = pe_abs > 500.0
    mid = ~(lo | hi)
    out[lo] = 1.0 - 0.5 * pe_abs[lo]
    out[hi] = 0.0
    out[mid] = pe_abs[mid] / np.expm1(pe_abs[mid])
    return out


class _Coo:
    def __init__(self, shape):
        self.shape = shape
        self.r, self.c, self.v = [], [], []

    def add(self, rows, cols, vals):
        self.r.append(np.asarray(rows).ravel())
        self.c.append(np.asarray(cols).ravel())
        self.v.append(np.asarray(vals).ravel())

    def csc(self):
        N = self.shape[0]
        if not self.r:
            return sp.csc_matrix((N, N))
        return sp.csc_matrix((np.concatenate(self.v),
                              (np.concatenate(self.r), np.concatenate(self.c))),
                             shape=self.shape)


def _face_rate(K_l, K_r, kmeander, u_face, adv_l, adv_r, d, split):
    """Patankar face rates (1/s) on a face of spacing d (convdiff.py:101-124)."""
    K_face = 2.0 * K_l * K_r / (K_l + K_r + 1e-30)
    if not split:
        K_face = K_face + kmeander
    D = K_face / d
    safe_K = np.where(K_face > 1e-30, K_face, 1e-30)
    pe = np.minimum(np.abs(u_face * d / safe_K), 500.0)
    diff = D * patankar_A(pe) / d
    return diff + adv_l, diff + adv_r


def _wrap_face(g, split):
    """Face rates and terrain ratios of the periodic wrap face between column
    nx-1 (L) and column 0 (R) (convdiff.py:150-202)."""
    d = np.broadcast_to(g.dx[None, :], (g.nz, g.ny))
    uw = g.u_wrap
    up = g.u_plus_wrap if split else np.maximum(uw, 0.0)
    um = g.u_minus_wrap if split else np.maximum(-uw, 0.0)
    km = g.kmu_wrap if g.kmu_wrap is not None else np.zeros_like(uw)
    rl, rr = _face_rate(g.kxxyy[:, :, -1], g.kxxyy[:, :, 0], km, uw, up / d, um / d, d, split)
    pl, pr = g.dP[:, :, -1], g.dP[:, :, 0]
    face = 0.5 * (pl + pr)
    ok = (pl > 0) & (pr > 0)
    return rl, rr, np.where(ok, face / pr, 1.0), np.where(ok, face / pl, 1.0)


def horizontal_convdiff(g):
    """Pressure-form horizontal block T_hcd (convdiff.py:42-387)."""
    nz, ny, nx = g.nz, g.ny, g.nx
    N = nz * ny * nx
    idx = np.arange(N).reshape(nz, ny, nx)
    dx3 = np.broadcast_to(g.dx[None, :, None], (nz, ny, nx))
    diag = np.zeros((nz, ny, nx))
    coo = _Coo((N, N))
    split = g.split
    up_all = g.u_plus if split else np.maximum(g.u, 0.0)
    um_all = g.u_minus if split else np.maximum(-g.u, 0.0)
    vp_all = g.v_plus if split else np.maximum(g.v, 0.0)
    vm_all = g.v_minus if split else np.maximum(-g.v, 0.0)
    if nx > 1:
        d = dx3[:, :, 1:]
        rl, rr = _face_rate(g.kxxyy[:, :, :-1], g.kxxyy[:, :, 1:], g.kmu[:, :, 1:],
                            g.u[:, :, 1:], up_all[:, :, 1:] / d, um_all[:, :, 1:] / d, d, split)
        pl, pr = g.dP[:, :, :-1], g.dP[:, :, 1:]
        face = 0.5 * (pl + pr)
        ok = (pl > 0) & (pr > 0)
        trr = np.where(ok, face / pr, 1.0)
        trl = np.where(ok, face / pl, 1.0)
        diag[:, :, 1:] += rr * trr
        coo.add(idx[:, :, 1:], idx[:, :, :-1], -(rl * trr))
        diag[:, :, :-1] += rl * trl
        coo.add(idx[:, :, :-1], idx[:, :, 1:], -(rr * trl))
    if getattr(g, "periodic_lon", False) and nx > 1:
        # wrap face (convdiff.py:150-202): cell 0 is R, cell nx-1 is L
        rl, rr, trr, trl = _wrap_face(g, split)
        diag[:, :, 0] += rr * trr
        coo.add(idx[:, :, 0], idx[:, :, -1], -(rl * trr))
        diag[:, :, -1] += rl * trl
        coo.add(idx[:, :, -1], idx[:, :, 0], -(rr * trl))
    else:
        diag += lateral_boundary_loss(g, x_only=True).reshape(nz, ny, nx)
    dy = g.dy
    if ny > 1:
        rl, rr = _face_rate(g.kxxyy[:, :-1, :], g.kxxyy[:, 1:, :], g.kmv[:, 1:, :],
                            g.v[:, 1:, :], vp_all[:, 1:, :] / dy, vm_all[:, 1:, :] / dy, dy, split)
        ps, pn = g.dP[:, :-1, :], g.dP[:, 1:, :]
        face = 0.5 * (ps + pn)
        dxs, dxn = dx3[:, :-1, :], dx3[:, 1:, :]
        dxf = 0.5 * (dxs + dxn)
        ok = (ps > 0) & (pn > 0)
        trn = np.where(ok, (dxf / dxn) * (face / pn), 1.0)
        trs = np.where(ok, (dxf / dxs) * (face / ps), 1.0)
        diag[:, 1:, :] += rr * trn
        coo.add(idx[:, 1:, :], idx[:, :-1, :], -(rl * trn))
        diag[:, :-1, :] += rl * trs
        coo.add(idx[:, :-1, :], idx[:, 1:, :], -(rr * trs))
    # open y boundaries with the outer-face dx correction (convdiff.py:290-359)
    diag += lateral_boundary_loss(g, y_only=True).reshape(nz, ny, nx)
    pos = diag > 0
    coo.add(idx[pos], idx[pos], diag[pos])
    return coo.csc()


def lateral_boundary_loss(g, x_only=False, y_only=False):
    """Open-outflow loss rate of the lateral edge cells, (N,) (operator.py:25-178;
    the same terms as the boundary diagonals of convdiff.py:204-359): west
    u- and east outer-face u+ (non-periodic grids only), south v- and north
    outer-face v+ with the outer-face dx ratio."""
    nz, ny, nx = g.nz, g.ny, g.nx
    split = g.split
    loss = np.zeros((nz, ny, nx))
    dx3 = np.broadcast_to(g.dx[None, :, None], (nz, ny, nx))
    if not y_only and not (getattr(g, "periodic_lon", False) and nx > 1):
        w_out = g.u_minus[:, :, 0] if split else np.maximum(-g.u[:, :, 0], 0.0)
        loss[:, :, 0] += np.where(w_out > 0, w_out / dx3[:, :, 0], 0.0)
        e_out = (g.u_plus_e if split else g.u_e)
        e_cond = e_out > 0 if split else e_out >= 0
        loss[:, :, -1] += np.where(e_cond, e_out / dx3[:, :, -1], 0.0)
    if not x_only:
        dy = g.dy
        lat_s = g.lat[0] - g.dlat / 2.0
        lat_n = g.lat[-1] + g.dlat / 2.0
        tr_s = EARTH_RADIUS * np.cos(lat_s * DEG_TO_RAD) * g.dlon * DEG_TO_RAD / g.dx[0]
        tr_n = EARTH_RADIUS * np.cos(lat_n * DEG_TO_RAD) * g.dlon * DEG_TO_RAD / g.dx[-1]
        s_out = g.v_minus[:, 0, :] if split else np.maximum(-g.v[:, 0, :], 0.0)
        loss[:, 0, :] += np.where(s_out > 0, s_out / dy * tr_s, 0.0)
        n_out = (g.v_plus_n if split else g.v_n)
        n_cond = n_out > 0 if split else n_out >= 0
        loss[:, -1, :] += np.where(n_cond, n_out / dy * tr_n, 0.0)
    return loss.reshape(-1)


def vertical_advection(g):
    """Interface-flux upwind vertical advection (advection.py:383-523)."""
    nz, ny, nx = g.nz, g.ny, g.nx
    N = nz * ny * nx
    idx = np.arange(N).reshape(nz, ny, nx)
    wp = g.w_plus.copy()
    wm = g.w_minus.copy()
    wp[0] = 0.0
    wm[0] = 0.0
    dP = g.dP
    ok = dP > 0
    sdP = np.where(ok, dP, 1.0)
    diag = np.zeros((nz, ny, nx))
    coo = _Coo((N, N))
    # bottom face of k (k >= 1): downward = loss, upward = gain from k-1
    bot_dn = wp[:nz]
    bot_up = wm[:nz]
    has_below = np.zeros((nz, ny, nx), bool)
    has_below[1:] = True
    diag += np.where(ok & has_below & (bot_dn > 0), bot_dn / sdP, 0.0)
    m = ok & has_below & (bot_up > 0)
    kk, jj, ii = np.nonzero(m)
    coo.add(idx[kk, jj, ii], idx[kk - 1, jj, ii], -bot_up[m] / sdP[m])
    # top face of k: downward = gain from k+1 (none at domain top), upward = loss
    top_dn = wp[1:]
    top_up = wm[1:]
    has_above = np.zeros((nz, ny, nx), bool)
    has_above[:-1] = True
    m = ok & has_above & (top_dn > 0)
    kk, jj, ii = np.nonzero(m)
    coo.add(idx[kk, jj, ii], idx[kk + 1, jj, ii], -top_dn[m] / sdP[m])
    diag += np.where(ok & (top_up > 0), top_up / sdP, 0.0)
    pos = diag > 0
    coo.add(idx[pos], idx[pos], diag[pos])
    return coo.csc()


def vertical_diffusion(g):
    """Harmonic-mean K_zz with rho_face/rho_cell reweighting (mixing.py:14-117)."""
    nz, ny, nx = g.nz, g.ny, g.nx
    N = nz * ny * nx
    idx = np.arange(N).reshape(nz, ny, nx)
    Dz, dP, K = g.Dz, g.dP, g.kzz
    sDz = np.where(Dz > 0, Dz, 1.0)
    rho = np.where((Dz > 0) & (dP > 0), dP / (GRAVITY * sDz), 0.0)
    diag = np.zeros((nz, ny, nx))
    coo = _Coo((N, N))
    for k in range(nz - 1):
        a, b = Dz[k], Dz[k + 1]
        ok = (a > 0) & (b > 0)
        Kf = np.where(ok, 2.0 * K[k] * K[k + 1] / (K[k] + K[k + 1] + 1e-30), 0.0)
        dist = np.where(ok, 0.5 * (a + b), 1.0)
        r0, r1 = rho[k], rho[k + 1]
        rf = 0.5 * (r0 + r1)
        both = ok & (r0 > 0) & (r1 > 0)
        q0 = np.where(both, rf / np.where(r0 > 0, r0, 1.0), 1.0)
        q1 = np.where(both, rf / np.where(r1 > 0, r1, 1.0), 1.0)
        c0 = np.where(ok, Kf / (np.where(a > 0, a, 1.0) * dist) * q0, 0.0)
        c1 = np.where(ok, Kf / (np.where(b > 0, b, 1.0) * dist) * q1, 0.0)
        coo.add(idx[k][ok], idx[k + 1][ok], -c0[ok])
        coo.add(idx[k + 1][ok], idx[k][ok], -c1[ok])
        diag[k][ok] += c0[ok]
        diag[k + 1][ok] += c1[ok]
    pos = diag > 0
    coo.add(idx[pos], idx[pos], diag[pos])
    return coo.csc()


def cmfmc_transport(g):
    """Convective updraft + compensating subsidence (convection.py:25-140)."""
    nz, ny, nx = g.nz, g.ny, g.nx
    N = nz * ny * nx
    if g.cmfmc.size == 0:
        return sp.csc_matrix((N, N))
    idx = np.arange(N).reshape(nz, ny, nx)
    Dz, dP = g.Dz, g.dP
    sDz = np.where(Dz > 0, Dz, 1.0)
    rho = dP / (GRAVITY * sDz)
    srho = np.where(rho > 0, rho, 1.0)
    ok = (Dz > 0) & (dP > 0)
    diag = np.zeros((nz, ny, nx))
    coo = _Coo((N, N))
    for k in range(nz):
        F = np.maximum(g.cmfmc[k + 1], 0.0)
        act = ok[k] & (F > 0)
        if not act.any():
            continue
        src = np.where(act, F / (srho[k] * sDz[k]), 0.0)
        diag[k] += src
        if k < nz - 1:
            gain = act & ok[k + 1]
            if gain.any():
                sDz1 = np.where(Dz[k + 1] > 0, Dz[k + 1], 1.0)
                rec = np.where(gain, F / (srho[k + 1] * sDz1), 0.0)
                coo.add(idx[k + 1][gain], idx[k][gain], -rec[gain])
                diag[k + 1] += rec
                coo.add(idx[k][gain], idx[k + 1][gain], -src[gain])
    pos = diag > 0
    coo.add(idx[pos], idx[pos], diag[pos])
    return coo.csc()


def transport_block(g, concentration_form=None):
    """T = T_hcd + T_vadv + T_vdiff + T_conv, then diag(rho) T diag(1/rho) when
    the grid is in concentration form (operator.py:281-353, the
    ``concentration_state`` switch at operator.py:341)."""
    if concentration_form is None:
        concentration_form = bool(getattr(g, "concentration_state", True))
    T = horizontal_convdiff(g) + vertical_advection(g) + vertical_diffusion(g) + cmfmc_transport(g)
    if concentration_form:
        rho = g.rho().reshape(-1)
        T = (sp.diags(rho) @ T @ sp.diags(1.0 / rho)).tocsc()
    return T.tocsc()


def species_operator(T, sink_diag):
    """L_s = T + diag(d_s) (operator.py:572-585, deposition.py:101-146)."""
    N = T.shape[0]
    return (T + sp.diags(np.asarray(sink_diag, dtype=np.float64), 0, shape=(N, N))).tocsc()


def mass_balance_diagnostics(grids):
    """|row sum| of the transport block per day over laterally interior cells
    (operator.py:598-652)."""
    DAY = 86400.0
    nz, ny, nx = grids[0].nz, grids[0].ny, grids[0].nx
    inner = np.zeros((nz, ny, nx), bool)
    inner[:, 1:-1, 1:-1] = True
    ri_l, rt_l, per = [], [], []
    for g in grids:
        T = transport_block(g)
        w = g.state_weights().reshape(-1)  # rho, or 1 in the pressure form (operator.py:626)
        r = (np.asarray(T @ w).ravel() / w).reshape(nz, ny, nx) * DAY
        r = np.where(inner, r, np.nan)
        ri_l.append(r[:-1].ravel())
        rt_l.append(r[-1].ravel())
        per.append(r)
    ri = np.abs(np.concatenate(ri_l))
    ri = ri[np.isfinite(ri)]
    rt = np.abs(np.concatenate(rt_l))
    rt = rt[np.isfinite(rt)]
    pl = np.abs(np.stack(per))
    return {
        "interior_median": float(np.median(ri)),
        "interior_p90": float(np.percentile(ri, 90)),
        "interior_p99": float(np.percentile(ri, 99)),
        "interior_max": float(ri.max()),
        "interior_frac_above_0.01": float(np.mean(ri > 0.01)),
        "interior_frac_above_0.1": float(np.mean(ri > 0.1)),
        "top_median": float(np.median(rt)),
        "top_p90": float(np.percentile(rt, 90)),
        "layer_p90": [float(np.nanpercentile(pl[:, k], 90)) for k in range(nz)],
        "layer_mean_signed": [float(np.nanmean(np.stack(per)[:, k])) for k in range(nz)],
    }
