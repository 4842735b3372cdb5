"""Generate golden vectors by running the reference ORBIT code itself.

Run in a container where the reference checkout is importable (its default
location is used unless ORBIT_REFERENCE is set):

    python tests/golden/make_golden.py                   # every golden file
    python tests/golden/make_golden.py --pressure-form   # only pressure_form.npz
    python tests/golden/make_golden.py --species         # only species_ops.npz
    python tests/golden/make_golden.py --closure         # only closure.npz
    python tests/golden/make_golden.py --periodic        # only periodic.npz
    python tests/golden/make_golden.py --nox             # only nox_rate.npz

It builds reference ``GridData`` objects from this repository's seeded
synthetic meteorology (``orbit_b200.synthetic``), calls the reference's own
assembly, FCT, mass-balance and SuperLU periodic-orbit solvers, and stores
inputs and outputs in small ``.npz`` files beside this script.  The tests
compare the CPU oracle (``oracle/``) and the CUDA path against them; nothing
reads the reference at test time.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.environ.get("ORBIT_REFERENCE", "/root/reference"))

import scipy.sparse as sp  # noqa: E402

from orbit.core.grid_data import GridData, _compute_geometry, _compute_terrain_ratios  # noqa: E402
from orbit.core.indexing import CellIndexer  # noqa: E402
from orbit.core import convdiff, advection, mixing, convection, operator, fct  # noqa: E402
from orbit.core.deposition import assemble_deposition, IDX_PM25  # noqa: E402
from orbit.core.orbit import _factor_one_bin, solve_orbit_one_species, DTAU, N_BINS  # noqa: E402
from orbit.core.orbit_adjoint import solve_orbit_adjoint_one_species  # noqa: E402

from orbit_b200 import synthetic  # noqa: E402


def to_griddata(m: synthetic.MetBin, vd=None, wet=None) -> GridData:
    g = GridData()
    g.concentration_state = bool(m.concentration_state)
    g.nz, g.ny, g.nx = m.nz, m.ny, m.nx
    g.lat, g.lon, g.dlat, g.dlon = m.lat.copy(), m.lon.copy(), m.dlat, m.dlon
    g.dP, g.Dz = m.dP.copy(), m.Dz.copy()
    g.UAvg, g.VAvg = m.u.copy(), m.v.copy()
    g.UAvg_plus, g.UAvg_minus = m.u_plus.copy(), m.u_minus.copy()
    g.VAvg_plus, g.VAvg_minus = m.v_plus.copy(), m.v_minus.copy()
    g.has_split_fluxes = bool(m.split)
    g.U_face_e, g.U_plus_face_e, g.U_minus_face_e = m.u_e.copy(), m.u_plus_e.copy(), m.u_minus_e.copy()
    g.V_face_n, g.V_plus_face_n, g.V_minus_face_n = m.v_n.copy(), m.v_plus_n.copy(), m.v_minus_n.copy()
    g.Kzz, g.Kxxyy = m.kzz.copy(), m.kxxyy.copy()
    g.K_meander_u, g.K_meander_v = m.kmu.copy(), m.kmv.copy()
    w = m.w_plus - m.w_minus
    g.omega_edge, g.omega_edge_plus, g.omega_edge_minus = w, m.w_plus.copy(), m.w_minus.copy()
    g.has_interface_omega = True
    g.CMFMC = m.cmfmc.copy()
    g.periodic_lon = bool(m.periodic_lon)
    if m.periodic_lon:
        g.UAvg_wrap = m.u_wrap.copy()
        g.UAvg_plus_wrap, g.UAvg_minus_wrap = m.u_plus_wrap.copy(), m.u_minus_wrap.copy()
        g.K_meander_u_wrap = m.kmu_wrap.copy()
    z = np.zeros((m.nz, m.ny, m.nx))
    pdd = z.copy()
    if vd is not None:
        pdd[0] = vd
    g.particle_dry_dep = pdd
    g.particle_wet_dep = z.copy() if wet is None else wet.copy()
    _compute_geometry(g)
    _compute_terrain_ratios(g)
    return g


def met_arrays(prefix, m):
    out = {}
    for name in ("dP", "Dz", "u", "v", "u_plus", "u_minus", "v_plus", "v_minus", "u_e",
                 "u_plus_e", "u_minus_e", "v_n", "v_plus_n", "v_minus_n", "kxxyy", "kzz",
                 "w_plus", "w_minus", "cmfmc", "kmu", "kmv", "lat", "lon"):
        out[f"{prefix}{name}"] = getattr(m, name)
    out[f"{prefix}meta"] = np.array([m.nz, m.ny, m.nx, m.dlat, m.dlon, float(m.split)])
    if m.periodic_lon:
        for name in ("u_wrap", "u_plus_wrap", "u_minus_wrap", "kmu_wrap"):
            out[f"{prefix}{name}"] = getattr(m, name)
    return out


def csc_arrays(prefix, M):
    M = M.tocsc()
    M.sum_duplicates()
    M.sort_indices()
    return {f"{prefix}data": M.data, f"{prefix}indices": M.indices, f"{prefix}indptr": M.indptr}


def main():
    rng = np.random.default_rng(7)
    # ---- assembly + FCT + mass-balance goldens on a small terrain grid ----
    nz, ny, nx = 5, 8, 9
    met = [synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=3000.0, rho_profile=True,
                                  cmfmc_frac=0.3, wind_std=6.0) for _ in range(N_BINS)]
    # non-split variant with a face-centred meander diffusivity
    ns = synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=3000.0, rho_profile=True,
                                cmfmc_frac=0.3, split=False)
    ns.kmu = rng.uniform(0.0, 500.0, (nz, ny, nx))
    ns.kmv = rng.uniform(0.0, 500.0, (nz, ny, nx))
    idx = CellIndexer(nz, ny, nx)
    sp_f = synthetic.make_species(11, nz, ny, nx)
    sp_f.wet[:] = rng.uniform(0.0, 2e-5, sp_f.wet.shape)
    out = {}
    for t, m in enumerate(met):
        out.update(met_arrays(f"met{t}_", m))
    out.update(met_arrays("ns_", ns))
    out["vd"], out["wet"], out["loss"], out["emis"] = sp_f.vd, sp_f.wet, sp_f.loss, sp_f.emis
    grids = [to_griddata(m, sp_f.vd[t], sp_f.wet[t]) for t, m in enumerate(met)]
    for t, g in enumerate(grids):
        T = operator.assemble_transport_block(g, idx)
        out.update(csc_arrays(f"T{t}_", T))
        D = assemble_deposition(g, idx, IDX_PM25, partitioning="equilibrium")
        out[f"D{t}"] = D.diagonal()
    gns = to_griddata(ns)
    out.update(csc_arrays("Tns_hcd_", convdiff.assemble_horizontal_convdiff(gns, idx)))
    out.update(csc_arrays("T0_hcd_", convdiff.assemble_horizontal_convdiff(grids[0], idx)))
    out.update(csc_arrays("T0_vadv_", advection.assemble_vertical_advection(grids[0], idx)))
    out.update(csc_arrays("T0_vdiff_", mixing.assemble_vertical_diffusion(grids[0], idx)))
    out.update(csc_arrays("T0_conv_", convection.assemble_cmfmc_transport(grids[0], idx)))
    pe = np.concatenate([[0.0, 1e-8, 1e-7, 1e-6, 2e-6], np.logspace(-5, 2.7, 40), [499.0, 500.0, 600.0]])
    out["pe"] = pe
    out["patankar"] = convdiff._patankar_A(pe.copy())
    mb = operator.mass_balance_diagnostics(grids, idx)
    out["mb_keys"] = np.array(["interior_median", "interior_p90", "interior_p99", "interior_max",
                               "interior_frac_above_0.01", "interior_frac_above_0.1",
                               "top_median", "top_p90"])
    out["mb_vals"] = np.array([mb[k] for k in out["mb_keys"]])
    out["mb_layer_p90"] = np.array(mb["layer_p90"])
    # FCT on a smooth positive field with extrema
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = (1.0 + np.sin(0.9 * ii) * np.cos(0.7 * jj) + 0.3 * kk + rng.random((nz, ny, nx))) * 1e-9
    c = c.reshape(-1)
    out["fct_c"] = c
    for t in range(2):
        out[f"fct_d{t}"] = fct.compute_horizontal_fct_source(grids[t], idx, c, DTAU)
        out[f"fct_d{t}_unlim"] = fct.compute_horizontal_fct_source(grids[t], idx, c, DTAU, limited=False)
    out.update(csc_arrays("fct_L0_", fct.assemble_fct_linear_operator(grids[0], idx, c, DTAU)))
    out["fct_dns"] = fct.compute_horizontal_fct_source(gns, idx, c, DTAU)

    # ---- orbit + adjoint goldens (SuperLU, tol 1e-12) ----
    I_N = sp.eye(idx.N, format="csc")
    L = []
    for t, g in enumerate(grids):
        T = operator.assemble_transport_block(g, idx)
        D = assemble_deposition(g, idx, IDX_PM25, partitioning="equilibrium")
        L.append((T + D + sp.diags(sp_f.loss[t].reshape(-1))).tocsc())
    lus = [_factor_one_bin(Lt, I_N, None, None) for Lt in L]
    e_list = [sp_f.emis[t] for t in range(N_BINS)]
    orbit, info = solve_orbit_one_species(lus, e_list, DTAU, tol=1e-12, maxiter=200)
    out["orbit"] = np.stack(orbit)
    out["orbit_info"] = np.array([info["gmres_iters"], info["residual"], info["periodicity"],
                                  info["neg_frac"]])
    R = [rng.random(idx.N) * (t + 1) for t in range(N_BINS)]
    adj, ainfo = solve_orbit_adjoint_one_species(lus, R, tol=1e-12)
    out["adj_R"] = np.stack(R)
    out["adjoint"] = np.stack(adj)
    out["adjoint_info"] = np.array([ainfo["gmres_iters"], ainfo["residual"], ainfo["periodicity"]])
    v = rng.standard_normal(idx.N)
    out["mono_v"] = v
    x = v.copy()
    for t in range(N_BINS):
        x = lus[t].solve(x)
    out["mono_Mv"] = x
    x = v.copy()
    for t in range(N_BINS - 1, -1, -1):
        x = lus[t].solve(x, trans="T")
    out["mono_MTv"] = x
    path = os.path.join(HERE, "small_grid.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes; gmres iters", info["gmres_iters"],
          "adj iters", ainfo["gmres_iters"])


def pressure_form():
    """Goldens of a grid in the pressure form (GridData.concentration_state
    False): the reference then keeps the assembled block as it is
    (operator.py:341), weights the FCT state and the mass-balance rows by 1
    (fct.py:451-456, operator.py:626)."""
    rng = np.random.default_rng(23)
    nz, ny, nx = 4, 7, 8
    m = synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=2000.0, rho_profile=True,
                               cmfmc_frac=0.3, wind_std=6.0)
    m.concentration_state = False
    idx = CellIndexer(nz, ny, nx)
    g = to_griddata(m)
    out = met_arrays("pf_", m)
    out.update(csc_arrays("pf_T_", operator.assemble_transport_block(g, idx)))
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = ((1.0 + np.sin(0.8 * ii) * np.cos(0.6 * jj) + 0.2 * kk + rng.random((nz, ny, nx))) * 1e-9).reshape(-1)
    out["pf_c"] = c
    out["pf_fct_d"] = fct.compute_horizontal_fct_source(g, idx, c, DTAU)
    out["pf_fct_d_unlim"] = fct.compute_horizontal_fct_source(g, idx, c, DTAU, limited=False)
    out.update(csc_arrays("pf_fct_L_", fct.assemble_fct_linear_operator(g, idx, c, DTAU)))
    mb = operator.mass_balance_diagnostics([g], idx)
    keys = ["interior_median", "interior_p90", "interior_p99", "interior_max", "top_median", "top_p90"]
    out["pf_mb_keys"] = np.array(keys)
    out["pf_mb_vals"] = np.array([mb[k] for k in keys])
    path = os.path.join(HERE, "pressure_form.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


SPECIES_FIELDS = ("particle_dry_dep", "NH3_dry_dep", "SO2_dry_dep", "NOx_dry_dep", "HNO3_dry_dep", "O3_dry_dep",
                  "VOC_dry_dep", "particle_wet_dep", "other_gas_wet_dep", "SO2_wet_dep", "NHPartitioning",
                  "NHPartitioningEq", "NO3Partitioning", "NO3PartitioningEq", "SO2oxidation", "archive_OH",
                  "j_no2_soa", "is_land", "F_p_vbs", "F_p_vbs_surface")


def species_operators():
    """Goldens of assemble_species_operators (operator.py:371-595) on two grids:
    'full' carries every optional field (HNO3/O3/VOC dry deposition, land
    mask, both partition fractions, VBS particle fractions, j(NO2) with the
    photolytic sink on, archive OH for the aging cascade, NOx/O3/CO rates);
    'min' only the required ones (fallback velocities, zero NO3 fraction,
    pure-particle VBS, no aging, SO2 rate by override)."""
    rng = np.random.default_rng(41)
    nz, ny, nx = 4, 6, 7
    idx = CellIndexer(nz, ny, nx)
    N = idx.N
    m = synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=1000.0, rho_profile=True, cmfmc_frac=0.3)
    out = met_arrays("sp_", m)

    def u(lo, hi, shape):
        return rng.uniform(lo, hi, shape)

    full = {"particle_dry_dep": u(1e-4, 5e-3, (nz, ny, nx)), "NH3_dry_dep": u(1e-3, 2e-2, (nz, ny, nx)),
            "SO2_dry_dep": u(1e-3, 1e-2, (nz, ny, nx)), "NOx_dry_dep": u(1e-4, 3e-3, (nz, ny, nx)),
            "HNO3_dry_dep": u(1e-2, 5e-2, (nz, ny, nx)), "O3_dry_dep": u(5e-4, 8e-3, (nz, ny, nx)),
            "VOC_dry_dep": u(5e-4, 3e-3, (nz, ny, nx)), "particle_wet_dep": u(0, 2e-5, (nz, ny, nx)),
            "other_gas_wet_dep": u(0, 5e-5, (nz, ny, nx)), "SO2_wet_dep": u(0, 3e-5, (nz, ny, nx)),
            "NHPartitioning": u(0, 1, (nz, ny, nx)), "NHPartitioningEq": u(0, 1, (nz, ny, nx)),
            "NO3Partitioning": u(0, 1, (nz, ny, nx)), "NO3PartitioningEq": u(0, 1, (nz, ny, nx)),
            "SO2oxidation": u(1e-7, 1e-5, (nz, ny, nx)), "archive_OH": u(1e5, 5e6, (nz, ny, nx)),
            "j_no2_soa": u(0, 8e-3, (nz, ny, nx)), "is_land": (rng.random((ny, nx)) > 0.3).astype(np.float64),
            "F_p_vbs": u(-0.1, 1.1, (5, nz, ny, nx)), "F_p_vbs_surface": u(0, 1, (5, ny, nx))}
    rates = {"nox_to_no3_rate": u(1e-7, 1e-5, (nz, ny, nx)), "o3_loss_rate": u(1e-7, 1e-5, (nz, ny, nx)),
             "co_loss_rate": u(1e-8, 1e-6, (nz, ny, nx))}
    minimal = {k: full[k] for k in ("particle_dry_dep", "NH3_dry_dep", "SO2_dry_dep", "NOx_dry_dep",
                                    "particle_wet_dep", "other_gas_wet_dep", "SO2_wet_dep", "NHPartitioning")}
    so2_override = u(1e-7, 1e-5, (nz, ny, nx))
    for k, v in full.items():
        out[f"full_{k}"] = v
    for k, v in rates.items():
        out[f"rate_{k}"] = v
    out["so2_override"] = so2_override
    os.environ["ORBIT_VBS_A_PHOTO"] = "4.0e-4"
    for tag, fields, kw in (("full", full, rates), ("min", minimal, {"so2_ox_rate": so2_override})):
        g = to_griddata(m)
        for k, v in fields.items():
            setattr(g, k, v.copy())
        for part in ("marginal", "equilibrium"):
            res = operator.assemble_species_operators(g, idx, verbose=False, return_D_per_species=True,
                                                      partitioning=part, **kw)
            L, K, T, d, D, Kage = res
            key = f"{tag}_{part}"
            out[f"{key}_d"] = d
            out[f"{key}_D"] = np.stack([np.asarray(x.diagonal()) for x in D])
            out[f"{key}_Kkeys"] = np.array(sorted(K.keys()), dtype=np.int64).reshape(-1, 2)
            out[f"{key}_Kdiag"] = np.stack([np.asarray(K[k].diagonal()) for k in sorted(K.keys())])
            out[f"{key}_Kagekeys"] = np.array(sorted(Kage.keys()), dtype=np.int64)
            out[f"{key}_Kage"] = (np.stack([np.asarray(Kage[k].diagonal()) for k in sorted(Kage.keys())])
                                  if Kage else np.zeros((0, N)))
            L1 = L[1].tocsc()
            L1.sum_duplicates()
            L1.sort_indices()
            out.update(csc_arrays(f"{key}_L1_", L1))
            out.update(csc_arrays(f"{key}_T_", T))
    del os.environ["ORBIT_VBS_A_PHOTO"]
    path = os.path.join(HERE, "species_ops.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def closure():
    """Goldens of the closure loop's pieces: IsorropiaLUT.query
    (isorropia_lut.py:116-147) on a small synthetic 7-D table written in the
    reference's file layout (points inside, on grid nodes and outside the
    axes, where the reference extrapolates), and an AndersonAccelerator
    (closure_iteration.py:568-694) sequence with the safeguard on a linear
    fixed-point map."""
    import tempfile
    from orbit.core.isorropia_lut import IsorropiaLUT
    from orbit.core.closure_iteration import AndersonAccelerator
    rng = np.random.default_rng(57)
    axes = {"so4_axis": np.array([0.0, 1.0, 4.0, 10.0]), "nh_axis": np.array([0.0, 2.0, 8.0]),
            "no3_axis": np.array([0.0, 3.0, 9.0]), "ca_axis": np.array([0.0, 0.5]),
            "na_axis": np.array([0.0, 0.3]), "t_axis": np.array([260.0, 280.0, 300.0]),
            "rh_axis": np.array([0.1, 0.4, 0.7, 0.95])}
    shape = tuple(len(a) for a in axes.values())
    fields = {"f_nh4": rng.uniform(-0.1, 1.1, shape).astype(np.float32),
              "f_no3": rng.uniform(-0.1, 1.1, shape).astype(np.float32),
              "aerosol_water": rng.uniform(-1.0, 50.0, shape).astype(np.float32),
              "ph": rng.uniform(1.0, 6.0, shape).astype(np.float32)}
    out = {f"lut_{k}": v for k, v in {**axes, **fields}.items()}
    lo = np.array([a[0] for a in axes.values()])
    hi = np.array([a[-1] for a in axes.values()])
    pts = lo + (hi - lo) * rng.uniform(-0.15, 1.15, (400, 7))
    nodes = np.stack([rng.choice(a, 50) for a in axes.values()], axis=1)
    pts = np.concatenate([pts, nodes])
    out["lut_pts"] = pts
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "lut.npz")
        np.savez(path, **axes, **fields)
        os.environ["ORBIT_LUT_CACHE_DIR"] = os.path.join(tmp, "cache")
        lut = IsorropiaLUT(path, fields=("f_nh4", "f_no3", "aerosol_water", "ph"))
        res = lut.query(*[pts[:, d] for d in range(7)])
        lut2 = IsorropiaLUT(path)
        res2 = lut2.query(*[pts[:, d] for d in range(7)])
        del os.environ["ORBIT_LUT_CACHE_DIR"]
    out["lut_out"] = np.stack(res)
    out["lut_out_two_fields"] = np.stack(res2)
    # Anderson on g(x) = A x + b with A of spectral radius 0.9
    n = 40
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Q @ np.diag(rng.uniform(-0.9, 0.9, n)) @ Q.T
    b = rng.standard_normal(n)
    out["and_A"], out["and_b"] = A, b
    for tag, kw in (("m3", dict(m=3, beta=1.0)), ("m2d", dict(m=2, beta=0.6, safeguard_factor=1.05))):
        acc = AndersonAccelerator(**kw)
        x = np.zeros(n)
        xs, flags = [x.copy()], []
        for _ in range(10):
            x, ok = acc.apply_with_safeguard(x, A @ x + b)
            xs.append(x.copy())
            flags.append(ok)
        out[f"and_{tag}_x"] = np.stack(xs)
        out[f"and_{tag}_ok"] = np.array(flags)
        acc2 = AndersonAccelerator(**{k: v for k, v in kw.items() if k != "safeguard_factor"})
        x = np.zeros(n)
        xs = [x.copy()]
        for _ in range(10):
            x = acc2.update(x, A @ x + b)
            xs.append(x.copy())
        out[f"and_{tag}_x_unguarded"] = np.stack(xs)
    path = os.path.join(HERE, "closure.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def periodic():
    """Goldens of periodic-longitude grids (GridData.periodic_lon): the
    transport block with its wrap face (convdiff.py:150-202) in the split and
    the non-split (meander) flux modes, the lateral boundary loss of
    assemble_transport_block(..., return_boundary_fluxes=True) for a periodic
    and a regional grid (operator.py:25-178, 344-347), the FCT source of a
    periodic grid, the FCT source of regional grids with and without a
    lateral-inflow (ghost) field, and one periodic orbit solved by the
    reference's SuperLU path at tol 1e-12."""
    rng = np.random.default_rng(31)
    nz, ny, nx = 4, 6, 10
    out = {}
    for tag, split in (("ps_", True), ("pn_", False)):
        m = synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=1500.0, rho_profile=True, cmfmc_frac=0.3,
                                   wind_std=6.0, split=split, periodic=True)
        if not split:
            m.kmu = rng.uniform(0.0, 500.0, (nz, ny, nx))
            m.kmu_wrap = rng.uniform(0.0, 500.0, (nz, ny))
        idx = CellIndexer(nz, ny, nx)
        g = to_griddata(m)
        out.update(met_arrays(tag, m))
        T, loss = operator.assemble_transport_block(g, idx, return_boundary_fluxes=True)
        out.update(csc_arrays(f"{tag}T_", T))
        out[f"{tag}loss"] = np.asarray(loss)
        kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        c = ((1.0 + np.sin(0.7 * ii) * np.cos(0.5 * jj) + 0.2 * kk + rng.random((nz, ny, nx))) * 1e-9).reshape(-1)
        out[f"{tag}c"] = c
        out[f"{tag}fct_d"] = fct.compute_horizontal_fct_source(g, idx, c, DTAU)
    # lateral loss of a regional grid (split and non-split)
    for tag, split in (("rs_", True), ("rn_", False)):
        m = synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=1500.0, rho_profile=True, wind_std=6.0,
                                   split=split)
        g = to_griddata(m)
        out.update(met_arrays(tag, m))
        idx = CellIndexer(nz, ny, nx)
        _, loss = operator.assemble_transport_block(g, idx, return_boundary_fluxes=True)
        out[f"{tag}loss"] = np.asarray(loss)
        # FCT with a lateral-inflow field (fct.py:459-492 with c_ghost_flat)
        kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        c = ((1.0 + np.cos(0.9 * ii) * np.sin(0.4 * jj) + 0.1 * kk + rng.random((nz, ny, nx))) * 1e-9).reshape(-1)
        cg = (rng.uniform(0.2, 3.0, (nz, ny, nx)) * 1e-9).reshape(-1)
        out[f"{tag}c"], out[f"{tag}cg"] = c, cg
        out[f"{tag}fct_dg"] = fct.compute_horizontal_fct_source(g, idx, c, DTAU, c_ghost_flat=cg)
        out[f"{tag}fct_dg_unlim"] = fct.compute_horizontal_fct_source(g, idx, c, DTAU, limited=False,
                                                                      c_ghost_flat=cg)
        out[f"{tag}fct_d"] = fct.compute_horizontal_fct_source(g, idx, c, DTAU)
    # one periodic orbit (eight periodic bins, one species)
    met = [synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=1500.0, rho_profile=True, cmfmc_frac=0.3,
                                  wind_std=6.0, periodic=True) for _ in range(N_BINS)]
    spc = synthetic.make_species(4111, nz, ny, nx)
    d = spc.sink_diag(met)
    idx = CellIndexer(nz, ny, nx)
    N = nz * ny * nx
    I_N = sp.identity(N, format="csc")
    lus = []
    for t, m in enumerate(met):
        out.update(met_arrays(f"om{t}_", m))
        T = operator.assemble_transport_block(to_griddata(m), idx)
        L = (T + sp.diags(d[t])).tocsc()
        lus.append(_factor_one_bin(L, I_N, None, None))
    orbit, info = solve_orbit_one_species(lus, [spc.emis[t] for t in range(N_BINS)], DTAU, tol=1e-12, maxiter=200)
    out["o_vd"], out["o_wet"], out["o_loss"], out["o_emis"] = spc.vd, spc.wet, spc.loss, spc.emis
    out["o_orbit"] = np.stack(orbit)
    path = os.path.join(HERE, "periodic.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes; gmres iters", info["gmres_iters"])


def nox_rate():
    """Goldens of build_nox_to_no3_rate (nox_to_no3_rate.py:94-155): every
    oxidant and aerosol field present, day and night channels; without NO,
    NO3 radical and the optional aerosol fields; with the night channel off."""
    from types import SimpleNamespace
    from orbit.core.nox_to_no3_rate import build_nox_to_no3_rate
    rng = np.random.default_rng(41)
    nz, ny, nx = 4, 5, 6
    sh = (nz, ny, nx)
    full = dict(Temperature=rng.uniform(220.0, 305.0, sh), Pressure=rng.uniform(2.0e4, 1.02e5, sh),
                archive_OH=rng.uniform(1e4, 1e7, sh), archive_NO=rng.uniform(0.0, 5.0, sh),
                archive_NO2=rng.uniform(0.0, 20.0, sh), archive_NO3rad=rng.uniform(0.0, 0.05, sh),
                pS=rng.uniform(0.0, 3.0, sh), pNH=rng.uniform(0.0, 2.0, sh), pNO=rng.uniform(0.0, 2.0, sh),
                dust_fine=rng.uniform(0.0, 10.0, sh), sea_salt_fine=rng.uniform(0.0, 5.0, sh))
    full["archive_NO2"][0, 0, :3] = 0.0  # NOx = 0 cells
    full["archive_NO"][0, 0, :3] = 0.0
    empty = np.array([])
    cases = {"full": dict(full),
             "lean": dict(full, archive_NO=empty, archive_NO3rad=empty, pNO=empty, dust_fine=empty)}
    out = {}
    for k, v in full.items():
        out[f"nx_{k}"] = v
    for tag, fields in cases.items():
        g = GridData()
        g.nz, g.ny, g.nx = nz, ny, nx
        for k, v in fields.items():
            setattr(g, k, v)
        out[f"nx_rate_{tag}"] = build_nox_to_no3_rate(g)
        out[f"nx_rate_{tag}_day"] = build_nox_to_no3_rate(g, disable_night=True)
    path = os.path.join(HERE, "nox_rate.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    if "--nox" in sys.argv:
        nox_rate()
    elif "--periodic" in sys.argv:
        periodic()
    elif "--pressure-form" in sys.argv:
        pressure_form()
    elif "--species" in sys.argv:
        species_operators()
    elif "--closure" in sys.argv:
        closure()
    else:
        main()
        pressure_form()
        species_operators()
        closure()
        periodic()
        nox_rate()
