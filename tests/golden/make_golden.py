"""Generate golden vectors by running the reference ORBIT code itself.

Run in a container where the reference checkout is importable (its default
location is used unless ORBIT_REFERENCE is set):

    python tests/golden/make_golden.py

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
    g.periodic_lon = False
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


if __name__ == "__main__":
    main()
