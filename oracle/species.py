"""Oracle: species sink diagonals and source couplings (numpy).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates, for one
bin given as a namespace with the reference GridData field names:

* ``assemble_deposition``                 orbit/core/deposition.py:101-146
* ``_get_dry_dep_velocity_2d``            orbit/core/deposition.py:263-304
* ``_get_wet_dep_rate_3d``                orbit/core/deposition.py:307-360
* ``_get_soa_photolysis_rate_3d``         orbit/core/deposition.py:149-168
* ``_nh_partitioning`` / ``_get_no3_partitioning`` / ``_get_hno3_vd`` /
  ``_get_o3_vd``                          orbit/core/deposition.py:171-260
* the diagonal chemistry and aging blocks of
  ``assemble_species_operators``          orbit/core/operator.py:419-585
* ``build_nox_to_no3_rate``               orbit/core/nox_to_no3_rate.py:94-155
  with ``air_density``, ``k_OH_NO2``, ``Keq_N2O5``, ``mean_speed_N2O5``
                                          orbit/core/oxidants.py:142-206
"""
from __future__ import annotations

import numpy as np

VBS_BINS = (11, 10, 9, 0, 12)  # C01, C1, C10, C100, C1000
AGING = ((12, 0), (0, 9), (9, 10), (10, 11))  # (source, destination)
N_SPECIES = 14


def _f(g, name):
    a = getattr(g, name, None)
    if a is None:
        return None
    a = np.asarray(a, dtype=np.float64)
    return a if a.size else None


def diagonals(g, partitioning="marginal", a_photo=0.0, so2_ox=None, nox_ox=None, o3_loss=None, co_loss=None,
              k_age=4.0e-11, aging_gain=1.075, chemistry=True):
    """(d (14, N), couplings {(target, source): (N,)}, deposition-only D (14, N),
    aging losses {source: (N,)})."""
    nz, ny, nx = g.nz, g.ny, g.nx
    N = nz * ny * nx
    pw, gw, pd = _f(g, "particle_wet_dep"), _f(g, "other_gas_wet_dep"), _f(g, "particle_dry_dep")[0]
    nh = _f(g, "NHPartitioningEq") if partitioning == "equilibrium" else None
    nh = nh if nh is not None else _f(g, "NHPartitioning")
    order = ("NO3Partitioning", "NO3PartitioningEq") if partitioning == "marginal" else \
        ("NO3PartitioningEq", "NO3Partitioning")
    no3 = next((_f(g, k) for k in order if _f(g, k) is not None), np.zeros((nz, ny, nx)))
    fp = getattr(g, "F_p_vbs", None)
    fp = np.asarray(fp) if fp is not None and np.asarray(fp).shape[:1] == (5,) else None
    fps = getattr(g, "F_p_vbs_surface", None)
    fps = np.asarray(fps) if fps is not None and np.asarray(fps).shape[:1] == (5,) else None
    j = _f(g, "j_no2_soa")
    hno3 = _f(g, "HNO3_dry_dep")
    if hno3 is None:
        hno3 = np.zeros((nz, ny, nx))
        hno3[0] = 0.03
    o3 = _f(g, "O3_dry_dep")
    if o3 is None:
        land = _f(g, "is_land")
        land = land if land is not None else np.ones((ny, nx))
        o3 = np.zeros((nz, ny, nx))
        o3[0] = np.where(land > 0, 0.004, 0.0005)
    voc = _f(g, "VOC_dry_dep")
    voc0 = voc[0] if voc is not None else np.full((ny, nx), 1.0e-3)
    dz0 = g.Dz[0]
    D = np.zeros((N_SPECIES, N))
    for s in range(N_SPECIES):
        if s in VBS_BINS:
            b = VBS_BINS.index(s)
            wet = fp[b] * pw if fp is not None else pw.copy()
            vd = fps[b] * pd + (1.0 - fps[b]) * voc0 if fps is not None else pd
        elif s in (1, 13, 5):
            wet, vd = pw.copy(), pd
        elif s == 2:
            wet = (1.0 - nh) * gw + nh * pw
            vd = (1.0 - nh[0]) * _f(g, "NH3_dry_dep")[0] + nh[0] * pd
        elif s == 3:
            wet, vd = _f(g, "SO2_wet_dep").copy(), _f(g, "SO2_dry_dep")[0]
        elif s == 4:
            wet, vd = np.zeros((nz, ny, nx)), _f(g, "NOx_dry_dep")[0]
        elif s == 6:
            wet = (1.0 - no3) * gw + no3 * pw
            vd = (1.0 - no3[0]) * hno3[0] + no3[0] * pd
        elif s == 7:
            wet, vd = np.zeros((nz, ny, nx)), o3[0]
        else:
            wet, vd = np.zeros((nz, ny, nx)), np.zeros((ny, nx))
        dd = wet.copy()
        dd[0] += np.where(dz0 > 0, vd / np.where(dz0 > 0, dz0, 1.0), 0.0)
        if s in VBS_BINS and j is not None and a_photo > 0:
            dd = dd + a_photo * j * (fp[VBS_BINS.index(s)] if fp is not None else 1.0)
        D[s] = dd.reshape(-1)
    d = D.copy()
    K, Kage = {}, {}
    if not chemistry:
        return d, K, D, Kage
    so2 = so2_ox if so2_ox is not None else _f(g, "SO2oxidation")
    so2 = np.asarray(so2).reshape(-1) if so2 is not None else np.zeros(N)
    d[3] += so2
    K[(5, 3)] = -so2
    if nox_ox is not None:
        d[4] += np.asarray(nox_ox).reshape(-1)
        K[(6, 4)] = -np.asarray(nox_ox).reshape(-1)
    if o3_loss is not None:
        d[7] += np.asarray(o3_loss).reshape(-1)
    if co_loss is not None:
        d[8] += np.asarray(co_loss).reshape(-1)
    oh = _f(g, "archive_OH")
    if oh is not None:
        roh = (k_age * oh).reshape(-1)
        for src, dst in AGING:
            r = roh * (1.0 - np.clip(fp[VBS_BINS.index(src)], 0.0, 1.0).reshape(-1)) if fp is not None else roh
            d[src] += r
            Kage[src] = r
            K[(dst, src)] = -aging_gain * r
    return d, K, D, Kage


def nox_to_no3_rate(g, disable_night=False):
    """NOx -> TotalNO3 first-order rate (1/s): OH + NO2 by day, N2O5
    hydrolysis on fine aerosol by night; None without archive OH / NO2."""
    oh, no2 = _f(g, "archive_OH"), _f(g, "archive_NO2")
    if oh is None or no2 is None:
        return None
    NA, KB, R = 6.02214076e23, 1.380649e-23, 8.31446
    T, P = _f(g, "Temperature"), _f(g, "Pressure")
    M = P * NA / (R * T) * 1e-6
    no = _f(g, "archive_NO")
    no_m = no * 1e-9 * M if no is not None else np.zeros_like(oh)
    no2_m = no2 * 1e-9 * M
    nox = no_m + no2_m
    safe = np.where(nox > 0, nox, 1.0)
    f_no2 = np.where(nox > 0, no2_m / safe, 1.0)
    k0 = 1.8e-30 * (T / 298.0) ** (-3.0) * M
    ratio = k0 / 2.8e-11
    k_oh = (k0 / (1.0 + ratio)) * 0.6 ** (1.0 / (1.0 + np.log10(ratio) ** 2))
    k_day = k_oh * oh * f_no2
    k_night = np.zeros_like(k_day)
    no3 = _f(g, "archive_NO3rad")
    if not disable_night and no3 is not None:
        n2o5 = 5.8e-27 * np.exp(10840.0 / T) * no2_m * (no3 * 1e-9 * M)
        fine = np.zeros_like(T)
        for name, ratio_c in (("pS", 96.0632 / 32.0655), ("pNH", 18.03851 / 14.0067), ("pNO", 62.00501 / 14.0067),
                              ("dust_fine", 1.0), ("sea_salt_fine", 1.0)):
            a = _f(g, name)
            if a is not None:
                fine = fine + (a * ratio_c if ratio_c != 1.0 else a)
        area = fine * 1e-9 * (3.0 / (1700.0 * 0.15e-6)) * 1e-2
        v = np.sqrt(8.0 * KB * T / (np.pi * (108.01e-3 / NA))) * 100.0
        k_het = 0.25 * 0.02 * v * area
        k_night = np.where(nox > 0, 2.0 * k_het * n2o5 / safe, 0.0)
    return k_day + k_night
