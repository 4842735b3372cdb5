"""Drop-in for the reference's transport assembly and air-mass-balance gate
(orbit/core/operator.py).

``assemble_transport_block(grid, indexer)`` (operator.py:281-347) assembles
the concentration-form block on the device (K1) and returns it as the
reference does, a scipy CSC matrix; ``transport_stencil(grid)`` returns the
device-resident [7, N] stencil the factorization consumes directly.
``mass_balance_diagnostics(grids, indexer)`` (operator.py:598-652) computes
the row sums on the device (K7) and the same order statistics; ``gate``
applies the reference's abort rule (cli.py:1590-1615: p90 > tol aborts).
``assemble_species_operators(grid, indexer, ...)`` (operator.py:371-595)
computes the transport block (K1) and every species' sink diagonal and
source-coupling diagonal (K1b, one kernel per bin) on the device and returns
the reference's tuple of scipy matrices; ``species_diagonals_device`` keeps
them on the device for the factorization.
"""
from __future__ import annotations

import numpy as np

from .grid import met_from_griddata

MASS_BALANCE_TOL = 0.05  # per day (cli.py:161)

# Species indices and aging pairs of the reference inventory (deposition.py:54-106)
IDX_VBS_C100, IDX_PM25, IDX_TOTAL_NH, IDX_SO2, IDX_NOX, IDX_PSO4, IDX_TOTAL_NO3, IDX_O3, IDX_CO = range(9)
IDX_VBS_C10, IDX_VBS_C1, IDX_VBS_C01, IDX_VBS_C1000, IDX_POA = 9, 10, 11, 12, 13
N_SPECIES = 14
VBS_AGING_PAIRS = ((IDX_VBS_C1000, IDX_VBS_C100), (IDX_VBS_C100, IDX_VBS_C10), (IDX_VBS_C10, IDX_VBS_C1),
                   (IDX_VBS_C1, IDX_VBS_C01))


def transport_stencil(grid, with_rowsum=False):
    from . import device
    md = device.MetDevice(met_from_griddata(grid))
    return device.assemble_transport(md, with_rowsum=with_rowsum)


def _periodic(grid) -> bool:
    return bool(getattr(grid, "periodic_lon", False)) and int(grid.nx) > 1


def assemble_transport_block(grid, indexer=None, scheme: str = "exp", return_boundary_fluxes: bool = False):
    """The transport block as a scipy CSC matrix (K1 on the device); with
    ``return_boundary_fluxes`` also the lateral boundary loss rate of every
    cell (compute_lateral_boundary_loss, operator.py:25-178), as the
    reference returns them (operator.py:344-347)."""
    if scheme != "exp":
        raise ValueError(f"Only the Patankar exponential scheme is supported (got scheme={scheme!r})")
    from . import device
    md = device.MetDevice(met_from_griddata(grid))
    T = device.assemble_transport(md).cpu().numpy()
    Tc = device.stencil_to_csr(T, int(grid.nz), int(grid.ny), int(grid.nx), periodic=_periodic(grid)).tocsc()
    if not return_boundary_fluxes:
        return Tc
    return Tc, device.boundary_loss(md).cpu().numpy()


def species_operator(T, sink_diag):
    """L_s = T + diag(d_s) (operator.py:572-585) for a host CSC T."""
    import scipy.sparse as sp
    N = T.shape[0]
    return (T + sp.diags(np.asarray(sink_diag, dtype=np.float64), 0, shape=(N, N))).tocsc()


def mass_balance_diagnostics(grids, indexer=None, blocks=("transport",)) -> dict:
    from . import device
    mets = [device.MetDevice(met_from_griddata(g)) for g in grids]
    Ts = [device.assemble_transport(m) for m in mets]
    out = device.mass_balance(mets, Ts)
    out["units"] = "per day, |row sum| of the transport block, laterally interior cells, all bins"
    return out


def gate(diag: dict, tol: float = MASS_BALANCE_TOL) -> bool:
    """True when the air-mass balance passes (interior p90 <= tol per day)."""
    return not (diag["interior_p90"] > tol)


def _field(grid, name):
    a = getattr(grid, name, None)
    if a is None:
        return None
    a = np.asarray(a, dtype=np.float64)
    return a if a.size else None


def build_nox_to_no3_rate(grid, disable_night: bool = False):
    """Drop-in for orbit/core/nox_to_no3_rate.py::build_nox_to_no3_rate
    (94-155): the per-cell NOx -> TotalNO3 rate (1/s) from the grid's archive
    oxidants, computed on the device (K1b); None when archive_OH or
    archive_NO2 is empty, as the reference returns."""
    from . import device
    if _field(grid, "archive_OH") is None or _field(grid, "archive_NO2") is None:
        return None
    names = {"temperature": "Temperature", "pressure": "Pressure", "oh": "archive_OH", "no": "archive_NO",
             "no2": "archive_NO2", "no3rad": "archive_NO3rad", "p_s": "pS", "p_nh": "pNH", "p_no": "pNO",
             "dust_fine": "dust_fine", "sea_salt_fine": "sea_salt_fine"}
    f = {k: _field(grid, v) for k, v in names.items()}
    shape = (int(grid.nz), int(grid.ny), int(grid.nx))
    return device.nox_to_no3_rate(f, disable_night).cpu().numpy().reshape(shape)


def _partition_fields(grid, partitioning):
    """The TotalNH and TotalNO3 particle fractions the reference blends with
    (_nh_partitioning, _get_no3_partitioning: deposition.py:171-216)."""
    if partitioning not in ("marginal", "equilibrium"):
        raise ValueError(f"partitioning must be one of ('marginal', 'equilibrium'), got {partitioning!r}")
    nh = _field(grid, "NHPartitioningEq") if partitioning == "equilibrium" else None
    if nh is None:
        nh = _field(grid, "NHPartitioning")
    marg, eq = _field(grid, "NO3Partitioning"), _field(grid, "NO3PartitioningEq")
    order = (marg, eq) if partitioning == "marginal" else (eq, marg)
    no3 = next((f for f in order if f is not None), None)
    return nh, no3


def species_fields(grid, partitioning="marginal", so2_ox_rate=None, nox_to_no3_rate=None, o3_loss_rate=None,
                   co_loss_rate=None, chemistry=True):
    """Per-cell fields of ``orbit_species_diagonals`` from a reference GridData,
    with the reference's choices of optional fields and rates
    (operator.py:419-549, deposition.py:171-360); plus the scalars
    (a_photo, k_age, aging_gain).  ``chemistry=False`` leaves the chemistry
    loss terms out (the deposition-only diagonals D)."""
    import os
    nz, ny, nx = int(grid.nz), int(grid.ny), int(grid.nx)
    nh, no3 = _partition_fields(grid, partitioning)
    f = {"Dz": _field(grid, "Dz"), "particle_dry_dep": _field(grid, "particle_dry_dep"),
         "nh3_dry_dep": _field(grid, "NH3_dry_dep"), "so2_dry_dep": _field(grid, "SO2_dry_dep"),
         "nox_dry_dep": _field(grid, "NOx_dry_dep"), "hno3_dry_dep": _field(grid, "HNO3_dry_dep"),
         "o3_dry_dep": _field(grid, "O3_dry_dep"), "is_land": _field(grid, "is_land"),
         "voc_dry_dep": _field(grid, "VOC_dry_dep"), "particle_wet_dep": _field(grid, "particle_wet_dep"),
         "other_gas_wet_dep": _field(grid, "other_gas_wet_dep"), "so2_wet_dep": _field(grid, "SO2_wet_dep"),
         "nh_part": nh, "no3_part": no3}
    fp = getattr(grid, "F_p_vbs", None)
    f["fp_vbs"] = np.asarray(fp, dtype=np.float64) if fp is not None and np.asarray(fp).shape[:1] == (5,) else None
    fps = getattr(grid, "F_p_vbs_surface", None)
    f["fp_vbs_surface"] = (np.asarray(fps, dtype=np.float64)
                           if fps is not None and np.asarray(fps).shape[:1] == (5,) else None)
    a_photo = float(os.environ.get("ORBIT_VBS_A_PHOTO", 0.0))
    f["j_no2"] = _field(grid, "j_no2_soa") if a_photo > 0.0 else None
    k_age, gain = 0.0, 1.0
    if chemistry:
        f["so2_ox"] = (np.asarray(so2_ox_rate, dtype=np.float64).reshape(nz, ny, nx) if so2_ox_rate is not None
                       else _field(grid, "SO2oxidation"))
        oh = _field(grid, "archive_OH")
        if nox_to_no3_rate is None and oh is not None:
            nox_to_no3_rate = build_nox_to_no3_rate(grid)  # operator.py:474-476
        for key, rate in (("nox_ox", nox_to_no3_rate), ("o3_loss", o3_loss_rate), ("co_loss", co_loss_rate)):
            f[key] = np.asarray(rate, dtype=np.float64).reshape(nz, ny, nx) if rate is not None else None
        if oh is not None:
            if "ORBIT_VBS_FRAG" in os.environ:
                raise ValueError("ORBIT_VBS_FRAG was removed in 1.0.3; set ORBIT_VBS_AGING_GAIN (default 1.075) "
                                 "instead.")
            f["archive_oh"] = oh
            k_age = float(os.environ.get("ORBIT_VBS_K_AGE", "4.0e-11"))
            gain = float(os.environ.get("ORBIT_VBS_AGING_GAIN", "1.075"))
    missing = [k for k in ("Dz", "particle_dry_dep", "nh3_dry_dep", "so2_dry_dep", "nox_dry_dep",
                           "particle_wet_dep", "other_gas_wet_dep", "so2_wet_dep", "nh_part") if f.get(k) is None]
    if missing:
        raise ValueError(f"grid lacks the species fields {missing}")
    return f, a_photo, k_age, gain


def species_diagonals_device(grid, partitioning="marginal", **rates):
    """(14, N) sink diagonals and (6, N) coupling diagonals on the device (K1b)."""
    from . import device
    f, a_photo, k_age, gain = species_fields(grid, partitioning, **rates)
    return device.species_diagonals(int(grid.nz), int(grid.ny), int(grid.nx), f, a_photo, k_age, gain)


def assemble_species_operators(grid, indexer=None, verbose: bool = True, scheme: str = "exp",
                               nox_to_no3_rate=None, so2_ox_rate=None, o3_loss_rate=None, co_loss_rate=None,
                               return_D_per_species: bool = False, partitioning: str = "marginal"):
    """Device drop-in of assemble_species_operators (operator.py:371-595):
    returns (L_species, K_sources, T, d_species[, D, K_age_loss]) with the
    reference's types (scipy CSC matrices, a dict keyed (target, source), a
    (14, N) array).  The transport block (K1) and all diagonals (K1b) are
    computed on the device."""
    import scipy.sparse as sp
    from . import device
    if scheme != "exp":
        raise ValueError(f"Only scheme='exp' is supported (got {scheme!r})")
    nz, ny, nx = int(grid.nz), int(grid.ny), int(grid.nx)
    N = nz * ny * nx
    rates = dict(nox_to_no3_rate=nox_to_no3_rate, so2_ox_rate=so2_ox_rate, o3_loss_rate=o3_loss_rate,
                 co_loss_rate=co_loss_rate)
    f, a_photo, k_age, gain = species_fields(grid, partitioning, **rates)
    Tst = transport_stencil(grid).cpu().numpy()
    d, k = device.species_diagonals(nz, ny, nx, f, a_photo, k_age, gain)
    d = d.cpu().numpy()
    k = k.cpu().numpy()
    T = device.stencil_to_csr(Tst, nz, ny, nx, periodic=_periodic(grid)).tocsc()
    idx = np.arange(N)

    def diag(v):
        return sp.csc_matrix((v, (idx, idx)), shape=(N, N))

    K_sources = {(IDX_PSO4, IDX_SO2): diag(k[0])}
    if nox_to_no3_rate is not None:
        K_sources[(IDX_TOTAL_NO3, IDX_NOX)] = diag(k[1])
    aging = f.get("archive_oh") is not None
    if aging:
        for q, (src, dst) in enumerate(VBS_AGING_PAIRS):
            K_sources[(dst, src)] = diag(k[2 + q])
    L_species = []
    for s in range(N_SPECIES):
        st = Tst.copy()
        st[0] = st[0] + d[s]
        L_species.append(device.stencil_to_csr(st, nz, ny, nx, periodic=_periodic(grid)).tocsc())
    if verbose:
        print(f"{N_SPECIES} species operators on the device: {N:,} cells, couplings = {len(K_sources)}")
    if not return_D_per_species:
        return L_species, K_sources, T, d
    # deposition-only diagonals (chemistry off) and the aging losses
    f0, a0, _, _ = species_fields(grid, partitioning, chemistry=False)
    dd, _ = device.species_diagonals(nz, ny, nx, f0, a0, 0.0, 1.0)
    dd = dd.cpu().numpy()
    D = [diag(dd[s]) for s in range(N_SPECIES)]
    K_age_loss = {}
    if aging:
        _, kl = device.species_diagonals(nz, ny, nx, f, a_photo, k_age, -1.0)
        kl = kl.cpu().numpy()
        for q, (src, dst) in enumerate(VBS_AGING_PAIRS):
            K_age_loss[src] = diag(kl[2 + q])
    return L_species, K_sources, T, d, D, K_age_loss
