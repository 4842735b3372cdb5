/*
 * liborbit_b200 — C ABI of the B200-native periodic-orbit solver.
 *
 * Every entry point returns an int status (ORBIT_OK = 0); on failure
 * orbit_last_error() returns a message for the calling thread.  Device
 * buffers are caller-owned (plain device pointers plus sizes); handles
 * (symbolic analysis, factor batches) own their internal workspace and are
 * created and destroyed in matching pairs.  Each call takes the CUDA stream
 * to run on; distinct handles may be used from distinct threads at once.
 *
 * Index conventions: cell = k*ny*nx + j*nx + i (reference CellIndexer,
 * orbit/core/indexing.py:5-45); vectors passed in and out are in this cell
 * order.  Stencil arrays are [7][N] with directions
 * {centre, west, east, south, north, below, above}.
 *
 * Each declaration cites the reference interface it replaces.
 */
#ifndef ORBIT_B200_H_
#define ORBIT_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* orbit_stream_t; /* == cudaStream_t */

enum {
  ORBIT_OK = 0,
  ORBIT_ERR_ARG = 1,       /* bad argument (reference: ValueError) */
  ORBIT_ERR_NOMEM = 2,     /* device allocation failed */
  ORBIT_ERR_CUDA = 3,      /* CUDA runtime error */
  ORBIT_ERR_TIMEOUT = 4,   /* a bounded device spin-wait gave up */
  ORBIT_ERR_PIVOT = 5,     /* zero or non-finite pivot (reference: umfpack status != 0, solve.py:231) */
  ORBIT_ERR_NOCONV = 6,    /* GMRES hit maxiter (reference prints a WARNING, orbit.py:184) */
  ORBIT_ERR_INTERNAL = 7,
  ORBIT_ERR_NOTFINITE = 8  /* non-finite input or iterate */
};

enum { ORBIT_PREC_FP64 = 64, ORBIT_PREC_FP32 = 32 };

typedef struct orbit_symbolic_s* orbit_symbolic_t;
typedef struct orbit_factor_s* orbit_factor_t;

/* Message of the last failed call on this thread. */
const char* orbit_last_error(void);
/* Library version string. */
const char* orbit_version(void);
/* Number of CUDA kernels this library has launched since it was loaded.  No
 * reference counterpart (the reference runs no device code); used to account
 * for device work in benchmarks. */
long long orbit_kernel_launches(void);

/* Per-bin averaged meteorology on the device (each pointer nz*ny*nx doubles
 * unless noted).  Field meaning follows GridData, orbit/core/grid_data.py:19-215. */
typedef struct {
  const double* dP;
  const double* Dz;
  const double* u;        /* UAvg (west face of each cell) */
  const double* v;        /* VAvg (south face) */
  const double* u_plus;   /* UAvg_plus */
  const double* u_minus;  /* UAvg_minus */
  const double* v_plus;
  const double* v_minus;
  const double* u_e;      /* east outer face, (nz, ny) */
  const double* u_plus_e; /* (nz, ny) */
  const double* v_n;      /* north outer face, (nz, nx) */
  const double* v_plus_n; /* (nz, nx) */
  const double* kxxyy;
  const double* kzz;
  const double* w_plus;   /* interface downward flux, (nz+1, ny, nx) */
  const double* w_minus;  /* interface upward flux,   (nz+1, ny, nx) */
  const double* cmfmc;    /* (nz+1, ny, nx) or NULL */
  const double* kmu;      /* face meander K (non-split mode only) or NULL */
  const double* kmv;
  const double* lat;      /* (ny,) degrees */
  double dlat, dlon;      /* degrees */
  int split;              /* has_split_fluxes */
  int pressure_form;      /* 1 when GridData.concentration_state is False: the
                             transported variable is the mixing ratio, the state
                             weights are 1 and the transport block is not put in
                             concentration form (operator.py:341, fct.py:451-454,
                             operator.py:626); 0 (default) for the concentration form */
  int periodic_lon;       /* GridData.periodic_lon (nx >= 3): cells i = nx-1 and
                             i = 0 share the wrap face and the x-boundary loss is
                             absent (convdiff.py:150-216); the stencil's W entry of
                             i = 0 and E entry of i = nx-1 are the wrap couplings */
  const double* u_wrap;       /* UAvg_wrap, (nz, ny); periodic grids only */
  const double* u_plus_wrap;  /* UAvg_plus_wrap, (nz, ny); split mode */
  const double* u_minus_wrap; /* UAvg_minus_wrap, (nz, ny); split mode */
  const double* kmu_wrap;     /* K_meander_u_wrap, (nz, ny); non-split mode, may be NULL */
} orbit_met_t;

/* Symbolic analysis of one (nz, ny, nx) domain: geometric nested dissection
 * into dense supernodes plus the static factor/solve schedules.  Replaces
 * umfpack_symbolic / compute_metis_ordering (orbit/core/solve.py:88-207,
 * 299-335); like them it is computed once and reused for every species,
 * bin and met draw of the domain.  leaf_cells <= 0 selects the default. */
int orbit_symbolic_create(int nz, int ny, int nx, int leaf_cells, orbit_symbolic_t* out);
/* orbit_symbolic_create with every tuning option explicit (the autotuner's
 * search space): nested-dissection leaf size, solve chunk size (factor entries
 * per row chunk of the medium-batch schedule; the small- and large-batch
 * schedules use half and twice that), the smallest pivot count of a
 * tensor-core supernode, and the whole-subtree solve-task divisor (0 = none).
 * Values <= 0 (subtree_div < 0) take the ORBIT_B200_* environment setting or
 * the default.  Extends the ordering options of umfpack_symbolic
 * (orbit/core/solve.py:88-207: ordering, qinit). */
int orbit_symbolic_create_ex(int nz, int ny, int nx, int leaf_cells, int chunk_elems, int tc_min_n,
                             int subtree_div, orbit_symbolic_t* out);
/* orbit_symbolic_create_ex for a grid that may be periodic in longitude
 * (GridData.periodic_lon, orbit/core/grid_data.py:426-445; needs nx >= 3):
 * the pattern then has the wrap-face couplings of cells i = 0 and i = nx - 1
 * (convdiff.py:150-202), which the dissection separates by cutting the
 * longitude ring with two planes. */
int orbit_symbolic_create_grid(int nz, int ny, int nx, int periodic_x, int leaf_cells, int chunk_elems,
                               int tc_min_n, int subtree_div, orbit_symbolic_t* out);
/* Replaces umfpack_free_symbolic (orbit/core/solve.py:291-296). */
int orbit_symbolic_destroy(orbit_symbolic_t sym);
/* info[0..14] = N, nsuper, nlevels, factor nnz (sum n^2+2nm), factor
 * elements per instance, front elements per instance, max front, factor
 * flops, solve items per bin, update-vector length, leaf_cells, max n/m,
 * largest front inside a subtree solve task, floats of tensor-core operand
 * packs per fp32 instance, supernodes factored whole by one CTA each
 * (ORBIT_B200_FUSED_MAX_N, default 64, 0 = none). */
int orbit_symbolic_info(orbit_symbolic_t sym, int64_t* info, int n_info);
/* perm[new] = cell (host array of N int32). */
int orbit_symbolic_perm(orbit_symbolic_t sym, int32_t* perm_host);
/* Copy a named host array of the analysis (int32 or int64 elements, as the
 * analysis stores it) for inspection and host-side checks; dst may be NULL to
 * query *count.  Names: perm, iperm, first, n, m, parent, level, child, uoff,
 * uidx, rel, ldn, ldm, ldf, fac_off, front_off, level_front_size,
 * ent_level_off, ent_pos, ent_src, ginv, ginv_off, woff, sitems, phase_off, phase_offT,
 * nchunk_fwd, nchunk_bwd, nchunk_fwdT, nchunk_bwdT.  No reference counterpart
 * (UMFPACK's symbolic object is opaque); it exists so the structure can be
 * verified on a host without a GPU.  The analysis itself never touches the
 * device: device copies are made by the first orbit_factor_create. */
int orbit_symbolic_array(orbit_symbolic_t sym, const char* name, void* dst, int64_t capacity,
                         int64_t* count);

/* K1: assemble the concentration-form transport block T of one bin as a
 * 7-point stencil (device, [7][N] doubles), and the per-cell row sum of the
 * pressure-form block (device, N doubles, may be NULL).  Replaces
 * assemble_transport_block (orbit/core/operator.py:281-353) with its parts
 * assemble_horizontal_convdiff (convdiff.py:42-387),
 * assemble_vertical_advection (advection.py:383-523),
 * assemble_vertical_diffusion (mixing.py:14-117) and
 * assemble_cmfmc_transport (convection.py:25-140). */
int orbit_assemble_transport(int nz, int ny, int nx, const orbit_met_t* met,
                             double* T_stencil, double* rowsum, orbit_stream_t stream);
/* Lateral boundary loss rate of every cell (device, N doubles, >= 0, zero
 * inside the domain): the open-outflow terms of the transport block's
 * diagonal at the x (non-periodic grids) and y edges.  Replaces
 * compute_lateral_boundary_loss (orbit/core/operator.py:25-178), the second
 * result of assemble_transport_block(..., return_boundary_fluxes=True)
 * (operator.py:344-347). */
int orbit_transport_boundary_loss(int nz, int ny, int nx, const orbit_met_t* met, double* loss,
                                  orbit_stream_t stream);

/* Per-cell species fields of one bin for the species operators (device
 * pointers; (nz, ny, nx) doubles unless noted; NULL where marked optional).
 * Field meaning follows GridData (orbit/core/grid_data.py:19-215). */
typedef struct {
  const double* Dz;
  const double* particle_dry_dep;  /* dry-deposition velocities (m/s); layer 0 is read */
  const double* nh3_dry_dep;
  const double* so2_dry_dep;
  const double* nox_dry_dep;
  const double* hno3_dry_dep;      /* optional: 3 cm/s at the surface when NULL */
  const double* o3_dry_dep;        /* optional: 0.4 cm/s over land, 0.05 over water */
  const double* is_land;           /* optional (ny, nx): land everywhere when NULL */
  const double* voc_dry_dep;       /* optional: 0.1 cm/s organic vapour when NULL */
  const double* particle_wet_dep;  /* wet-deposition rates (1/s) */
  const double* other_gas_wet_dep;
  const double* so2_wet_dep;
  const double* nh_part;           /* TotalNH particle fraction (marginal or equilibrium, chosen by the caller) */
  const double* no3_part;          /* optional TotalNO3 particle fraction: 0 when NULL */
  const double* fp_vbs;            /* optional (5, nz, ny, nx) VBS particle fractions, bins C01..C1000 */
  const double* fp_vbs_surface;    /* optional (5, ny, nx) */
  const double* j_no2;             /* optional photolysis frequency for the SOA photolytic sink */
  double a_photo;                  /* its scaling A_PHOTO (0 = off) */
  const double* so2_ox;            /* optional SO2 -> pSO4 rate (1/s): 0 when NULL */
  const double* nox_ox;            /* optional NOx -> TotalNO3 rate */
  const double* o3_loss;           /* optional O3 chemistry loss */
  const double* co_loss;           /* optional CO chemistry loss */
  const double* archive_oh;        /* optional OH (molec/cm3): VBS aging when non-NULL */
  double k_age;                    /* aging rate constant (cm3/molec/s) */
  double aging_gain;               /* mass gained by the next-lower bin per unit aged */
} orbit_species_fields_t;

/* Oxidant fields of one bin for the archive-driven NOx -> TotalNO3 rate
 * (device pointers, (nz, ny, nx) doubles; NULL where marked optional).  Field
 * meaning follows GridData (orbit/core/grid_data.py:140-206). */
typedef struct {
  const double* temperature;   /* Temperature, K */
  const double* pressure;      /* Pressure, Pa (layer centre) */
  const double* oh;            /* archive_OH, molec/cm3 */
  const double* no;            /* archive_NO, ppbv; optional */
  const double* no2;           /* archive_NO2, ppbv */
  const double* no3rad;        /* archive_NO3rad, ppbv; optional (no night channel without it) */
  const double* p_s;           /* pS, ug/m3 of S; optional */
  const double* p_nh;          /* pNH, ug/m3 of N; optional */
  const double* p_no;          /* pNO, ug/m3 of N; optional */
  const double* dust_fine;     /* ug/m3; optional */
  const double* sea_salt_fine; /* ug/m3; optional */
} orbit_oxidant_fields_t;

/* K1b: the 14 species' diagonal sink rates d_s (wet deposition + surface
 * dry-deposition velocity / Dz + SOA photolysis + first-order chemistry
 * losses) and the diagonals of the six source couplings K[(target, source)]
 * (pSO4<-SO2, TotalNO3<-NOx, and the VBS aging cascade C100<-C1000,
 * C10<-C100, C1<-C10, C01<-C1), for one bin.  d: device (14, N); k_src:
 * device (6, N) or NULL, in that coupling order (rows of inactive couplings
 * are zero).  Replaces the diagonal parts of assemble_species_operators
 * (orbit/core/operator.py:371-595): assemble_deposition
 * (orbit/core/deposition.py:101-146, 263-360), the SO2 oxidation blocks
 * (orbit/core/chemistry.py:13-47) and the VBS aging blocks. */
/* Per-cell first-order NOx -> TotalNO3 rate (device, N doubles, 1/s): the
 * daytime OH + NO2 channel (JPL Troe rate times [OH] times the NO2 share of
 * NOx) plus, unless disable_night, N2O5 hydrolysis on fine aerosol (N2O5 in
 * thermal equilibrium with NO2 and the NO3 radical, uptake 0.02 on the
 * surface of 0.15 um spheres of the fine-mode mass).  Replaces
 * build_nox_to_no3_rate (orbit/core/nox_to_no3_rate.py:94-155, with
 * oxidants.py:142-206), which assemble_species_operators calls when a grid
 * carries archive OH and no rate is given (operator.py:474-476). */
int orbit_nox_to_no3_rate(int64_t n_cells, const orbit_oxidant_fields_t* f, int disable_night, double* rate,
                          orbit_stream_t stream);

int orbit_species_diagonals(int nz, int ny, int nx, const orbit_species_fields_t* fields, double* d,
                            double* k_src, orbit_stream_t stream);

/* Coupled right-hand sides of one target species for 8 bins:
 * out[tau] = e[tau] - sum_q kdiag[q][tau] * c_q[tau + shift_q] (c_q a source
 * orbit, (9, N) device; shift 0 = start-of-bin, 1 = end-of-bin coupling;
 * kdiag (n_src, 8, N) device; e, out (8, N) device, out may alias e).
 * Replaces the K @ c_src products of solve_orbit_all_species
 * (orbit/core/orbit.py:249-307) for the diagonal K-blocks of
 * assemble_species_operators. */
int orbit_source_coupling(int64_t N, int n_src, const double* const* c_src, const int* shift,
                          const double* kdiag, const double* e, double* out, orbit_stream_t stream);

/* K7: air-mass-balance row sums |T rho / rho| per day over laterally
 * interior cells for nbins stencils; writes the interior (nz-1 layers) and
 * top-layer magnitudes to out_interior / out_top (device, nbins*(nz-1)*(ny-2)*(nx-2)
 * and nbins*(ny-2)*(nx-2) doubles).  Replaces the row-sum part of
 * mass_balance_diagnostics (orbit/core/operator.py:598-652). */
int orbit_mass_balance_rows(int nz, int ny, int nx, int nbins, const double* const* T_stencils,
                            const double* const* rho, double* out_interior, double* out_top,
                            orbit_stream_t stream);

/* K2: limited horizontal FCT deferred-correction source d_AD for n_vec
 * concentration vectors on one bin's grid.  c and d are device (n_vec, N).
 * Replaces compute_horizontal_fct_source (orbit/core/fct.py:459-492). */
int orbit_fct_source(int nz, int ny, int nx, const orbit_met_t* met, int n_vec,
                     const double* c, double dt, int limited, double* d, orbit_stream_t stream);

/* The 7-D ISORROPIA lookup table on the device: seven ascending axes (total
 * SO4, total NH, total NO3, crustal Ca, sea-salt Na in ug/m3, T in K, RH in
 * 0-1; device doubles, at least two points each) and up to four float32
 * fields of shape n[0] x ... x n[6], C order (f_nh4, f_no3, aerosol_water,
 * ph; NULL where not loaded). */
typedef struct {
  const double* axis[7];
  int n[7];
  const float* field[4];
} orbit_lut_t;

/* Query the LUT at n_pts points (pts: device (7, n_pts), one row per axis):
 * multilinear interpolation, linear extrapolation from the edge cells, in
 * double precision; out: device (4, n_pts) = clip(f_nh4, 0, 1),
 * clip(f_no3, 0, 1), max(aerosol_water, 0), ph (NaN for fields not loaded).
 * Replaces IsorropiaLUT.query (orbit/core/isorropia_lut.py:116-147, scipy
 * RegularGridInterpolator "linear", fill_value None). */
int orbit_lut_query(const orbit_lut_t* lut, int64_t n_pts, const double* pts, double* out, orbit_stream_t stream);

/* out[i] = x_i . y for m <= 16 device vectors of n doubles (x: host array of
 * device pointers; out: host, m doubles; synchronizes the stream).  With
 * orbit_vec_combine, the device side of the Anderson step of the closure loop
 * (AndersonAccelerator.update, orbit/core/closure_iteration.py:568-694). */
int orbit_vec_dots(int64_t n, int m, const double* const* x, const double* y, double* out, orbit_stream_t stream);
/* y = beta y + sum_i coef[i] x_i for m <= 16 device vectors (coef: host; y may
 * be one of the x_i). */
int orbit_vec_combine(int64_t n, int m, const double* coef, const double* const* x, double beta, double* y,
                      orbit_stream_t stream);

/* Frozen-gain FCT tangent-linear operator L_AD of n_vec baseline
 * concentrations c_base (device, n_vec x N): per face the gain C * beta of the
 * baseline (Zalesak coefficient times van Leer reconstruction factor) over dx,
 * terrain-weighted, in concentration form, so that L_AD c_base = -d_AD(c_base).
 * Output: n_vec stencils in the 7-point layout of the transport blocks
 * (device, n_vec x 7 x N doubles; the vertical entries are zero), so
 * T + L_AD is a plain stencil sum that the factorization accepts.  Replaces
 * assemble_fct_linear_operator (orbit/core/fct.py:495-572). */
int orbit_fct_linear_operator(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c_base,
                              double dt, double* stencil, orbit_stream_t stream);

/* orbit_fct_source with a lateral-inflow field: c_ghost (device, n_vec x N,
 * one per vector) holds the boundary inflow concentration c_bc, whose values
 * in the edge cells stand for the cells beyond each lateral edge: the
 * far-upwind values of the edge faces (which then keep their van Leer
 * reconstruction instead of dropping to first order) and the outside
 * neighbours of the Zalesak bounds.  Replaces compute_horizontal_fct_source
 * with c_ghost_flat (orbit/core/fct.py:459-492, 283-292, 381-400). */
int orbit_fct_source_ghost(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c,
                           const double* c_ghost, double dt, int limited, double* d, orbit_stream_t stream);

/* y_v = beta y_v + alpha S_v x_v, or S_v^T x_v when trans, for n_vec 7-point
 * stencils (device, n_vec x 7 x N) and vectors (device, n_vec x N): the
 * products L_AD c_{tau+1} of the marginal FCT outer iteration and their
 * transposes (orbit/modes/marginal.py:627-635, orbit/modes/adjoint.py:540-566
 * apply the same operators as scipy CSC products). */
int orbit_stencil_apply(int nz, int ny, int nx, int n_vec, const double* stencils, const double* x, double alpha,
                        double beta, int trans, double* y, orbit_stream_t stream);
/* orbit_stencil_apply on a grid that may be periodic in longitude: with
 * periodic_x (nx >= 3) the W entry of a cell in column 0 couples it to
 * column nx - 1 and the E entry of column nx - 1 to column 0, the wrap-face
 * entries of assemble_horizontal_convdiff (convdiff.py:150-202). */
int orbit_stencil_apply_grid(int nz, int ny, int nx, int periodic_x, int n_vec, const double* stencils,
                             const double* x, double alpha, double beta, int trans, double* y,
                             orbit_stream_t stream);

/* K2 without device allocation, for callers that cannot allocate device
 * memory at the point where they apply the FCT correction (a host model that
 * owns its whole device-memory budget through its own pool, or a time loop
 * that must not stall on the synchronization cudaFree can cause).  Same inputs,
 * outputs and results as orbit_fct_source.  No counterpart in the reference.
 * The scratch (x = c/rho, R+, R-) is one static device array of 3 x 2^20
 * doubles (24 MiB) that every GPU loading this library holds until exit, so
 * n_vec*nz*ny*nx must be <= 1,048,576 (larger requests return ORBIT_ERR_ARG).
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  The address is cached per device
 * ordinal for the life of the process and does not survive a cudaDeviceReset
 * (or any teardown of the device's primary context): do not call this entry
 * point after one.  All calls share the array, so calls that overlap on the
 * GPU (different streams or threads) race: serialize them. */
int orbit_fct_source_noalloc(int nz, int ny, int nx, const orbit_met_t* met, int n_vec,
                             const double* c, double dt, int limited, double* d,
                             orbit_stream_t stream);

/* A batch of n_orbits x 8 numeric factorizations of A = I + dtau (T + diag(sink))
 * sharing one symbolic.  precision = ORBIT_PREC_FP64 or ORBIT_PREC_FP32.
 * Replaces _factor_one_bin / _UmfpackLU.__init__ (orbit/core/orbit.py:79-96,
 * orbit/core/solve.py:210-243). */
int orbit_factor_create(orbit_symbolic_t sym, int n_orbits, int precision, orbit_factor_t* out);
/* General form: n_orbits solve slots over n_sets factor sets of n_bins (8)
 * factorizations each; slot o uses set (o % n_sets) until orbit_factor_map
 * says otherwise, so many right-hand sides can share one operator (the
 * reference reuses one lu_list_8 for all marginal and adjoint right-hand
 * sides, orbit/modes/adjoint.py:573-583).  n_bins = 1 (with one slot and one
 * set) holds a single factorization: the per-bin LU object the reference's
 * _factor_one_bin returns (orbit/core/orbit.py:79-96). */
int orbit_factor_create_ex(orbit_symbolic_t sym, int n_orbits, int n_sets, int n_bins, int precision,
                           orbit_factor_t* out);
/* Factor set used by each solve slot (host array of n_orbits indices). */
int orbit_factor_map(orbit_factor_t f, const int32_t* set_of_orbit);
int orbit_factor_destroy(orbit_factor_t f);
/* Factor the first n_active factor sets.  T_stencils / sink_diags are host
 * arrays of n_active*n_bins device pointers (set-major, bin-minor); a sink
 * pointer may be NULL.  The stencils are copied; callers may free them after
 * the call returns (stream-ordered). */
int orbit_factor_numeric(orbit_factor_t f, int n_active, const double* const* T_stencils,
                         const double* const* sink_diags, double dtau, orbit_stream_t stream);
/* Per-launch timing of the chained-solve kernel and of numeric factorizations
 * (CUDA events on the caller's stream).  mode 1: enable and reset; 0: disable
 * and reset; 2: read into out[6] = {chain launches, chain ms, chain
 * algorithmic bytes (factor values read), factor calls, factor ms, factor
 * flops}.  Reading synchronizes the recorded events.  The reference reports
 * t_factor/t_solve wall times per species (orbit/core/orbit.py:331-383). */
int orbit_factor_profile(orbit_factor_t f, int mode, double* out);
/* Device bytes held by the factor handle (reference: numeric_bytes, solve.py:233-236). */
int orbit_factor_bytes(orbit_factor_t f, int64_t* numeric_bytes, int64_t* workspace_bytes);

/* K4: chained solves x <- P_tau x for tau in [tau0, tau1) (trans = 0), or
 * x <- P_tau^T x for tau = tau1-1 .. tau0 (trans = 1), for n_active orbits, one
 * persistent launch.  x_in, x_out: device (n_active, N) in cell order.  With
 * forcing (device (n_active, 8, N), may be NULL) the forward chain solves
 * P_tau (x + fscale e_tau) and the transposed chain adds fscale e_tau after each
 * P_tau^T.  Replaces lu.solve(b, trans) chains: apply_monodromy
 * (orbit.py:99-107), compute_s (orbit.py:110-120), apply_monodromy_adjoint
 * and compute_s_adjoint (orbit_adjoint.py:36-67).  For FP32 factors,
 * refine != 0 applies one FP64 iterative-refinement step per bin. */
int orbit_chain_apply(orbit_factor_t f, int n_active, int trans, int tau0, int tau1,
                      const double* x_in, double* x_out, const double* forcing, double fscale,
                      int refine, orbit_stream_t stream);

/* K5: batched periodic-orbit GMRES(restart) solves of (I - M) c0 = s for the
 * first n_active orbits of a factored batch.  e: device (n_active, 8, N)
 * emissions; c_warm: device (n_active, N) or NULL; orbit_out: device
 * (n_active, 9, N); info_out: host (n_active, 8) doubles = {gmres_iters,
 * residual, periodicity, neg_frac, converged, s_norm, outer_refinements,
 * matvecs}.  Mixed precision (FP32 factors) runs inner GMRES on the FP32
 * monodromy inside an FP64 outer refinement of the monodromy residual.
 * Replaces solve_orbit_one_species (orbit/core/orbit.py:123-210). */
int orbit_gmres_solve(orbit_factor_t f, int n_active, const double* e, double dtau,
                      const double* c_warm, double tol, int maxiter, int restart,
                      double* orbit_out, double* info_out, orbit_stream_t stream);

/* Self-test of the bounded device waits: one chained-solve launch whose first
 * task waits for a completion count that nothing reaches.  Returns
 * ORBIT_ERR_TIMEOUT when the wait gave up, the status word was read and every
 * block left (the context stays usable; the handle's status is reset).  No
 * reference counterpart (the reference has no device waits). */
int orbit_selftest_wait_timeout(orbit_factor_t f, orbit_stream_t stream);

/* Transposed periodic-orbit solve (I - M^T) lam0 = s_adj with receptors R
 * (device (n_active, 8, N)); adjoint_out (n_active, 9, N); info_out (n_active, 8)
 * as above.  Replaces solve_orbit_adjoint_one_species
 * (orbit/core/orbit_adjoint.py:70-144). */
int orbit_adjoint_gmres_solve(orbit_factor_t f, int n_active, const double* R,
                              const double* lam_warm, double tol, int maxiter, int restart,
                              double* adjoint_out, double* info_out, orbit_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* ORBIT_B200_H_ */
