// K2: Zalesak-limited horizontal FCT deferred-correction source.
//
// Replaces compute_horizontal_fct_source (orbit/core/fct.py:459-492) with its
// helpers _vanleer_phi (fct.py:235-247), _horizontal_antidiffusive
// (fct.py:256-357, with or without the lateral-inflow ghost field),
// _zalesak_2d (fct.py:381-447) and
// _net_antidiffusive_into_cells (fct.py:360-378).  Pass 1 computes, per cell,
// the Zalesak ratios R+/R- from the four face fluxes touching it and the
// 5-point bounds; pass 2 limits every face with the ratios of its two cells
// and forms d = -div(C A) times rho.  Face fluxes are recomputed where needed
// rather than stored (each needs at most four cells along its axis).
#include <cuda_runtime.h>

#include "common.cuh"

namespace orbit {

namespace {

constexpr double kEarthRadius = 6378137.0;
constexpr double kGravity = 9.80665;
constexpr double kDegToRad = 3.14159265358979323846 / 180.0;

struct FctGeom {
  orbit_met_t g;
  int nz, ny, nx;
  double dt;
  // optional lateral-inflow concentration per vector (c-space, same layout as
  // c): its edge-cell values stand for the cells beyond each lateral edge
  const double* ghost = nullptr;
};


// State weight of a cell: rho = dP / (g Dz) in the concentration form, 1 in the
// pressure form (_state_weights, fct.py:451-456).
__device__ __forceinline__ double rho_at(const orbit_met_t& g, int64_t c) {
  if (g.pressure_form) return 1.0;
  const double dP = g.dP[c], Dz = g.Dz[c];
  return (dP > 0.0 && Dz > 0.0) ? dP / (kGravity * Dz) : 1.0;
}

// Value beyond the edge at edge cell e, in x = c / rho.
__device__ __forceinline__ double ghost_x(const orbit_met_t& g, const double* gh, int64_t e) {
  return gh[e] / rho_at(g, e);
}

__device__ __forceinline__ double vl_phi(double up, double far, double down) {
  const double num = up - far;
  const double den = down - up;
  const bool tiny = fabs(den) < 1e-30;
  double r = num / (tiny ? 1e-30 : den);
  if (tiny) r = fabs(num) < 1e-30 ? 1.0 : 1e6;
  return (r + fabs(r)) / (1.0 + fabs(r));
}

__device__ __forceinline__ double dx_at(const orbit_met_t& g, int j) {
  return kEarthRadius * cos(g.lat[j] * kDegToRad) * g.dlon * kDegToRad;
}

// Face between lo = (k, j, i-1) [x] or (k, j-1, i) [y] and hi = cell index `hi`.
// Returns flux = A * inv and the terrain weights; valid flag.
struct Face {
  double flux, trL, trR, beta, inv;
  bool ok;
};

// gh: the ghost field of this vector or null (fct.py:283-292: with a ghost
// field the far-upwind value beyond an edge is the ghost value of the edge
// cell; without one the face drops to first order there).
__device__ Face x_face(const FctGeom& G, const double* x, int k, int j, int ihi, const double* gh) {
  const orbit_met_t& g = G.g;
  const int nx = G.nx;
  const int64_t base = ((int64_t)k * G.ny + j) * nx;
  const int64_t hi = base + ihi, lo = hi - 1;
  const double cL = x[lo], cR = x[hi];
  const double cLL = ihi - 1 > 0 ? x[lo - 1] : gh ? ghost_x(g, gh, lo) : cL;
  const double cRR = ihi < nx - 1 ? x[hi + 1] : gh ? ghost_x(g, gh, hi) : cR;
  double pL = vl_phi(cL, cLL, cR);
  double pR = vl_phi(cR, cRR, cL);
  if (!gh && ihi - 1 == 0) pL = 0.0;
  if (!gh && ihi == nx - 1) pR = 0.0;
  const double up = G.g.split ? g.u_plus[hi] : fmax(g.u[hi], 0.0);
  const double um = G.g.split ? g.u_minus[hi] : fmax(-g.u[hi], 0.0);
  const double beta = 0.5 * (up * pL + um * pR);
  const double A = beta * (cR - cL);
  const double d = dx_at(g, j);
  const double inv = 1.0 / (d > 0.0 ? d : 1.0);
  const double dl = g.dP[lo], dr = g.dP[hi];
  Face f;
  f.ok = dl > 0.0 && dr > 0.0;
  const double face = 0.5 * (dl + dr);
  f.trL = f.ok ? face / (dl > 0.0 ? dl : 1.0) : 1.0;
  f.trR = f.ok ? face / (dr > 0.0 ? dr : 1.0) : 1.0;
  f.flux = A * inv;
  f.beta = beta;
  f.inv = inv;
  return f;
}

__device__ Face y_face(const FctGeom& G, const double* x, int k, int jhi, int i, const double* gh) {
  const orbit_met_t& g = G.g;
  const int nx = G.nx, ny = G.ny;
  const int64_t hi = ((int64_t)k * ny + jhi) * nx + i, lo = hi - nx;
  const double cS = x[lo], cN = x[hi];
  const double cSS = jhi - 1 > 0 ? x[lo - nx] : gh ? ghost_x(g, gh, lo) : cS;
  const double cNN = jhi < ny - 1 ? x[hi + nx] : gh ? ghost_x(g, gh, hi) : cN;
  double pS = vl_phi(cS, cSS, cN);
  double pN = vl_phi(cN, cNN, cS);
  if (!gh && jhi - 1 == 0) pS = 0.0;
  if (!gh && jhi == ny - 1) pN = 0.0;
  const double vp = G.g.split ? g.v_plus[hi] : fmax(g.v[hi], 0.0);
  const double vm = G.g.split ? g.v_minus[hi] : fmax(-g.v[hi], 0.0);
  const double beta = 0.5 * (vp * pS + vm * pN);
  const double A = beta * (cN - cS);
  const double dy = kEarthRadius * g.dlat * kDegToRad;
  const double inv = 1.0 / (dy > 0.0 ? dy : 1.0);
  const double dxs = dx_at(g, jhi - 1), dxn = dx_at(g, jhi);
  const double dxf = 0.5 * (dxs + dxn);
  const double ds = g.dP[lo], dn = g.dP[hi];
  Face f;
  f.ok = ds > 0.0 && dn > 0.0;
  const double face = 0.5 * (ds + dn);
  f.trL = f.ok ? (dxf / (dxs > 0.0 ? dxs : 1.0)) * (face / (ds > 0.0 ? ds : 1.0)) : 1.0;
  f.trR = f.ok ? (dxf / (dxn > 0.0 ? dxn : 1.0)) * (face / (dn > 0.0 ? dn : 1.0)) : 1.0;
  f.flux = A * inv;
  f.beta = beta;
  f.inv = inv;
  return f;
}

// x = c / rho for all vectors
__global__ void k_fct_x(FctGeom G, const double* c, double* x, int64_t N) {
  const double* cv = c + (int64_t)blockIdx.y * N;
  double* xv = x + (int64_t)blockIdx.y * N;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (int64_t)gridDim.x * blockDim.x)
    xv[e] = cv[e] / rho_at(G.g, e);
}

__global__ void k_fct_ratio(FctGeom G, const double* x_all, double* Rp_all, double* Rm_all, int64_t N) {
  const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= N) return;
  const double* x = x_all + (int64_t)blockIdx.y * N;
  const double* gh = G.ghost ? G.ghost + (int64_t)blockIdx.y * N : nullptr;
  const int nx = G.nx, ny = G.ny;
  const int i = (int)(cell % nx), j = (int)((cell / nx) % ny), k = (int)(cell / ((int64_t)nx * ny));
  const double c = x[cell];
  double cmax = c, cmin = c;
  // beyond an edge: the edge cell's ghost value, or the cell itself (clamped)
  const double out = gh ? ghost_x(G.g, gh, cell) : c;
  const double w = i > 0 ? x[cell - 1] : out, e = i < nx - 1 ? x[cell + 1] : out;
  const double s = j > 0 ? x[cell - nx] : out, n = j < ny - 1 ? x[cell + nx] : out;
  cmax = fmax(fmax(fmax(cmax, w), fmax(e, s)), n);
  cmin = fmin(fmin(fmin(cmin, w), fmin(e, s)), n);
  double Pp = 0.0, Pm = 0.0;
  auto acc = [&](double into) {
    Pp += fmax(into, 0.0);
    Pm += fmax(-into, 0.0);
  };
  if (nx > 1) {
    if (i > 0) {
      Face f = x_face(G, x, k, j, i, gh);
      acc(f.ok ? f.trR * f.flux : 0.0);
    }
    if (i < nx - 1) {
      Face f = x_face(G, x, k, j, i + 1, gh);
      acc(f.ok ? -f.trL * f.flux : 0.0);
    }
  }
  if (ny > 1) {
    if (j > 0) {
      Face f = y_face(G, x, k, j, i, gh);
      acc(f.ok ? f.trR * f.flux : 0.0);
    }
    if (j < ny - 1) {
      Face f = y_face(G, x, k, j + 1, i, gh);
      acc(f.ok ? -f.trL * f.flux : 0.0);
    }
  }
  const double Qp = (cmax - c) / G.dt, Qm = (c - cmin) / G.dt;
  Rp_all[(int64_t)blockIdx.y * N + cell] = Pp > 0.0 ? fmin(1.0, Qp / Pp) : 0.0;
  Rm_all[(int64_t)blockIdx.y * N + cell] = Pm > 0.0 ? fmin(1.0, Qm / Pm) : 0.0;
}

__global__ void k_fct_div(FctGeom G, const double* x_all, const double* Rp_all, const double* Rm_all,
                          int limited, double* d_all, int64_t N) {
  const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= N) return;
  const double* x = x_all + (int64_t)blockIdx.y * N;
  const double* Rp = Rp_all + (int64_t)blockIdx.y * N;
  const double* Rm = Rm_all + (int64_t)blockIdx.y * N;
  const double* gh = G.ghost ? G.ghost + (int64_t)blockIdx.y * N : nullptr;
  const int nx = G.nx, ny = G.ny;
  const int i = (int)(cell % nx), j = (int)((cell / nx) % ny), k = (int)(cell / ((int64_t)nx * ny));
  auto limiter = [&](const Face& f, int64_t lo, int64_t hi) {
    if (!limited) return 1.0;
    const double into_hi = f.ok ? f.trR * f.flux : 0.0;
    double C = into_hi >= 0.0 ? fmin(Rp[hi], Rm[lo]) : fmin(Rm[hi], Rp[lo]);
    return fmin(fmax(C, 0.0), 1.0);
  };
  double d = 0.0;
  if (nx > 1) {
    if (i > 0) {
      Face f = x_face(G, x, k, j, i, gh);
      const double fl = limiter(f, cell - 1, cell) * f.flux;
      d += f.ok ? f.trR * fl : 0.0;
    }
    if (i < nx - 1) {
      Face f = x_face(G, x, k, j, i + 1, gh);
      const double fl = limiter(f, cell, cell + 1) * f.flux;
      d -= f.ok ? f.trL * fl : 0.0;
    }
  }
  if (ny > 1) {
    if (j > 0) {
      Face f = y_face(G, x, k, j, i, gh);
      const double fl = limiter(f, cell - nx, cell) * f.flux;
      d += f.ok ? f.trR * fl : 0.0;
    }
    if (j < ny - 1) {
      Face f = y_face(G, x, k, j + 1, i, gh);
      const double fl = limiter(f, cell, cell + nx) * f.flux;
      d -= f.ok ? f.trL * fl : 0.0;
    }
  }
  d_all[(int64_t)blockIdx.y * N + cell] = d * rho_at(G.g, cell);
}

// Frozen-gain linearisation of the limited flux (assemble_fct_linear_operator,
// orbit/core/fct.py:495-572): each face's gain w = C beta / dx (C the Zalesak
// coefficient and beta the van Leer reconstruction factor of the baseline),
// distributed with the terrain weights so that L_AD x = -div(w (x_R - x_L)),
// then the similarity diag(rho) L diag(1/rho).  Output: the 7-point stencil
// layout of the transport blocks (centre, W, E, S, N, below, above; the
// vertical entries are zero), so L_low + L_AD is a plain stencil sum.
__global__ void k_fct_linop(FctGeom G, const double* x_all, const double* Rp_all, const double* Rm_all,
                            double* st_all, int64_t N) {
  const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= N) return;
  const double* x = x_all + (int64_t)blockIdx.y * N;
  const double* Rp = Rp_all + (int64_t)blockIdx.y * N;
  const double* Rm = Rm_all + (int64_t)blockIdx.y * N;
  double* st = st_all + (int64_t)blockIdx.y * 7 * N;
  const double* gh = nullptr;  // the frozen operator has no ghost field (fct.py:495-572)
  const int nx = G.nx, ny = G.ny;
  const int i = (int)(cell % nx), j = (int)((cell / nx) % ny), k = (int)(cell / ((int64_t)nx * ny));
  auto gain = [&](const Face& f, int64_t lo, int64_t hi) {
    if (!f.ok) return 0.0;
    const double into_hi = f.trR * f.flux;
    const double C = into_hi >= 0.0 ? fmin(Rp[hi], Rm[lo]) : fmin(Rm[hi], Rp[lo]);
    return fmin(fmax(C, 0.0), 1.0) * f.beta * f.inv;
  };
  const double rp = rho_at(G.g, cell);
  double cen = 0.0, w = 0.0, e = 0.0, s = 0.0, n = 0.0;
  if (nx > 1) {
    if (i > 0) {  // west face: this cell is its high side
      const Face f = x_face(G, x, k, j, i, gh);
      const double wr = f.trR * gain(f, cell - 1, cell);
      cen -= wr;
      w = wr * rp / rho_at(G.g, cell - 1);
    }
    if (i < nx - 1) {  // east face: low side
      const Face f = x_face(G, x, k, j, i + 1, gh);
      const double wl = f.trL * gain(f, cell, cell + 1);
      cen -= wl;
      e = wl * rp / rho_at(G.g, cell + 1);
    }
  }
  if (ny > 1) {
    if (j > 0) {
      const Face f = y_face(G, x, k, j, i, gh);
      const double wr = f.trR * gain(f, cell - nx, cell);
      cen -= wr;
      s = wr * rp / rho_at(G.g, cell - nx);
    }
    if (j < ny - 1) {
      const Face f = y_face(G, x, k, j + 1, i, gh);
      const double wl = f.trL * gain(f, cell, cell + nx);
      cen -= wl;
      n = wl * rp / rho_at(G.g, cell + nx);
    }
  }
  st[cell] = cen;
  st[N + cell] = w;
  st[2 * N + cell] = e;
  st[3 * N + cell] = s;
  st[4 * N + cell] = n;
  st[5 * N + cell] = 0.0;
  st[6 * N + cell] = 0.0;
}

}  // namespace

int fct_source(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c, double dt,
               int limited, double* d, double* scratch, cudaStream_t st, const double* ghost = nullptr) {
  const int64_t N = (int64_t)nz * ny * nx;
  FctGeom G{*met, nz, ny, nx, dt, ghost};
  double* x = scratch;
  double* Rp = scratch + (int64_t)n_vec * N;
  double* Rm = Rp + (int64_t)n_vec * N;
  dim3 g((unsigned)((N + 127) / 128), n_vec);
  k_fct_x<<<g, 128, 0, st>>>(G, c, x, N);
  note_launch();
  if (limited) {
    k_fct_ratio<<<g, 128, 0, st>>>(G, x, Rp, Rm, N);
    note_launch();
  }
  k_fct_div<<<g, 128, 0, st>>>(G, x, Rp, Rm, limited, d, N);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

int fct_linear_operator(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c, double dt,
                        double* stencil, double* scratch, cudaStream_t st) {
  const int64_t N = (int64_t)nz * ny * nx;
  FctGeom G{*met, nz, ny, nx, dt};
  double* x = scratch;
  double* Rp = scratch + (int64_t)n_vec * N;
  double* Rm = Rp + (int64_t)n_vec * N;
  dim3 g((unsigned)((N + 127) / 128), n_vec);
  k_fct_x<<<g, 128, 0, st>>>(G, c, x, N);
  note_launch();
  k_fct_ratio<<<g, 128, 0, st>>>(G, x, Rp, Rm, N);
  note_launch();
  k_fct_linop<<<g, 128, 0, st>>>(G, x, Rp, Rm, stencil, N);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

}  // namespace orbit

// ---------------------------------------------------------------------------
// FCT source without any device allocation.
//
// Some callers cannot allocate device memory when they apply the correction:
// a host model that hands this library a fixed device-memory budget and owns
// every other byte through its own pool, or a time-stepping loop that must not
// stall on the implicit synchronization cudaFree may cause.  For them the
// three per-cell scratch arrays of the two FCT passes (x = c / rho and the
// Zalesak ratios R+ and R-) live in one file-scope device array instead of a
// stream-ordered allocation.  Every GPU that loads the library holds the
// array (kFctNoAllocMaxCells doubles x 3, 24 MiB) until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace orbit {

// n_vec * nz * ny * nx may not exceed this (e.g. 12 vectors of 86,400 cells).
constexpr int64_t kFctNoAllocMaxCells = int64_t(1) << 20;

static __device__ __align__(256) double g_fct_scratch[3 * kFctNoAllocMaxCells];

namespace {
std::mutex g_fct_scratch_mu;
constexpr int kMaxDevices = 64;
double* g_fct_scratch_ptr[kMaxDevices] = {nullptr};
}  // namespace

int fct_source_noalloc(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c,
                       double dt, int limited, double* d, cudaStream_t st) {
  const int64_t cells = (int64_t)nz * ny * nx * n_vec;
  if (cells > kFctNoAllocMaxCells) {
    set_last_error("orbit_fct_source_noalloc: n_vec*nz*ny*nx = " + std::to_string(cells) +
                   " exceeds the static scratch limit of " + std::to_string(kFctNoAllocMaxCells) +
                   " cells; split the vectors over several calls or use orbit_fct_source");
    return ORBIT_ERR_ARG;
  }
  int dev = 0;
  ORBIT_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error("orbit_fct_source_noalloc: device ordinal out of range");
    return ORBIT_ERR_ARG;
  }
  double* scratch = nullptr;
  {
    // The array's name is only a host-side stand-in for the symbol; its device
    // address is looked up once per device, with that device current.  The
    // cached address belongs to the device's current primary context: after a
    // cudaDeviceReset the module may load elsewhere, so the entry point must
    // not be called after one.
    std::lock_guard<std::mutex> lk(g_fct_scratch_mu);
    if (!g_fct_scratch_ptr[dev]) {
      void* p = nullptr;
      ORBIT_CUDA_TRY(cudaGetSymbolAddress(&p, g_fct_scratch));
      g_fct_scratch_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_fct_scratch_ptr[dev];
  }
  // x, R+ and R- are fully overwritten by the passes that produce them, so the
  // scratch needs no clearing between calls.
  return fct_source(nz, ny, nx, met, n_vec, c, dt, limited, d, scratch, st);
}

}  // namespace orbit
