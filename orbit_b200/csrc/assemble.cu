// K1: on-device assembly of the concentration-form transport block as a
// 7-point stencil, and K7: the air-mass-balance row sums.
//
// One thread per cell evaluates every face that touches the cell, in the
// reference's arithmetic:
//   horizontal Patankar exponential convection-diffusion with dP (and dx)
//   terrain weights and open outflow boundaries   orbit/core/convdiff.py:42-387
//   upwind interface mass flux, closed ground      orbit/core/advection.py:383-523
//   harmonic-mean K_zz with rho_face/rho_cell       orbit/core/mixing.py:14-117
//   convective updraft + compensating subsidence   orbit/core/convection.py:25-140
// then applies the similarity diag(rho) T diag(1/rho) (operator.py:341-353).
// Row sums of the pressure-form block (T w)/w are emitted for the mass-balance
// gate (operator.py:598-652).
#include <cuda_runtime.h>

#include "common.cuh"

namespace orbit {

namespace {

constexpr double kEarthRadius = 6378137.0;
constexpr double kGravity = 9.80665;
constexpr double kDegToRad = 3.14159265358979323846 / 180.0;

__device__ __forceinline__ double patankar(double pe) {
  if (pe < 1e-6) return 1.0 - 0.5 * pe;
  if (pe > 500.0) return 0.0;
  return pe / expm1(pe);
}

// Face rates (rate_L, rate_R) of a horizontal face (convdiff.py:101-124).
__device__ __forceinline__ void face_rates(double KL, double KR, double km, int split, double uf,
                                           double up, double um, double d, double& rl, double& rr) {
  double Kf = 2.0 * KL * KR / (KL + KR + 1e-30);
  if (!split) Kf = Kf + km;
  const double D = Kf / d;
  const double sK = Kf > 1e-30 ? Kf : 1e-30;
  double pe = fabs(uf * d / sK);
  pe = pe < 500.0 ? pe : 500.0;
  const double diff = D * patankar(pe) / d;
  rl = diff + up / d;
  rr = diff + um / d;
}

__device__ __forceinline__ double rho_of(double dP, double Dz) {
  return (dP > 0.0 && Dz > 0.0) ? dP / (kGravity * Dz) : 1.0;
}

__global__ void k_assemble(int nz, int ny, int nx, orbit_met_t g, double* __restrict__ Tst,
                           double* __restrict__ rowsum, double* __restrict__ lat_loss) {
  const int64_t NN = (int64_t)nz * ny * nx;
  const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= NN) return;
  const int i = (int)(cell % nx);
  const int j = (int)((cell / nx) % ny);
  const int k = (int)(cell / ((int64_t)nx * ny));
  const int64_t nxy = (int64_t)nx * ny;
  auto dx_at = [&](double lat) { return kEarthRadius * cos(lat * kDegToRad) * g.dlon * kDegToRad; };
  const double dx = dx_at(g.lat[j]);
  const double dy = kEarthRadius * g.dlat * kDegToRad;
  const int split = g.split;
  auto UP = [&](int64_t c) { return split ? g.u_plus[c] : fmax(g.u[c], 0.0); };
  auto UM = [&](int64_t c) { return split ? g.u_minus[c] : fmax(-g.u[c], 0.0); };
  auto VP = [&](int64_t c) { return split ? g.v_plus[c] : fmax(g.v[c], 0.0); };
  auto VM = [&](int64_t c) { return split ? g.v_minus[c] : fmax(-g.v[c], 0.0); };
  const double dPc = g.dP[cell];
  double diag = 0.0, oW = 0.0, oE = 0.0, oS = 0.0, oN = 0.0, oB = 0.0, oT = 0.0;
  double bloss = 0.0;  // open-outflow terms at the lateral edges (part of diag)
  const bool px = g.periodic_lon != 0;
  const int64_t ew = (int64_t)k * ny + j;  // (k, j) index of the wrap-face fields
  // ---- x faces ----
  if (px && i == 0) {  // wrap face (convdiff.py:150-202): this cell is R, cell nx-1 is L
    const int64_t L = cell + nx - 1;
    const double uw = g.u_wrap[ew];
    const double upw = split ? g.u_plus_wrap[ew] : fmax(uw, 0.0);
    const double umw = split ? g.u_minus_wrap[ew] : fmax(-uw, 0.0);
    double rl, rr;
    face_rates(g.kxxyy[L], g.kxxyy[cell], g.kmu_wrap ? g.kmu_wrap[ew] : 0.0, split, uw, upw, umw, dx, rl, rr);
    const double dPL = g.dP[L];
    const bool ok = dPL > 0.0 && dPc > 0.0;
    const double trR = ok ? 0.5 * (dPL + dPc) / dPc : 1.0;
    diag += rr * trR;
    oW = -(rl * trR);
  } else if (i > 0) {  // west face: this cell is R
    const int64_t L = cell - 1;
    double rl, rr;
    face_rates(g.kxxyy[L], g.kxxyy[cell], g.kmu ? g.kmu[cell] : 0.0, split, g.u[cell], UP(cell),
               UM(cell), dx, rl, rr);
    const double dPL = g.dP[L];
    const bool ok = dPL > 0.0 && dPc > 0.0;
    const double trR = ok ? 0.5 * (dPL + dPc) / dPc : 1.0;
    diag += rr * trR;
    oW = -(rl * trR);
  } else {
    const double um = UM(cell);
    if (um > 0.0) bloss += um / dx;
  }
  if (px && i == nx - 1) {  // wrap face: this cell is L, cell 0 is R
    const int64_t R = cell - (nx - 1);
    const double uw = g.u_wrap[ew];
    const double upw = split ? g.u_plus_wrap[ew] : fmax(uw, 0.0);
    const double umw = split ? g.u_minus_wrap[ew] : fmax(-uw, 0.0);
    double rl, rr;
    face_rates(g.kxxyy[cell], g.kxxyy[R], g.kmu_wrap ? g.kmu_wrap[ew] : 0.0, split, uw, upw, umw, dx, rl, rr);
    const double dPR = g.dP[R];
    const bool ok = dPc > 0.0 && dPR > 0.0;
    const double trL = ok ? 0.5 * (dPc + dPR) / dPc : 1.0;
    diag += rl * trL;
    oE = -(rr * trL);
  } else if (i < nx - 1) {  // east face: this cell is L
    const int64_t R = cell + 1;
    double rl, rr;
    face_rates(g.kxxyy[cell], g.kxxyy[R], g.kmu ? g.kmu[R] : 0.0, split, g.u[R], UP(R), UM(R), dx,
               rl, rr);
    const double dPR = g.dP[R];
    const bool ok = dPc > 0.0 && dPR > 0.0;
    const double trL = ok ? 0.5 * (dPc + dPR) / dPc : 1.0;
    diag += rl * trL;
    oE = -(rr * trL);
  } else {
    const int64_t e = (int64_t)k * ny + j;
    if (split) {
      const double up = g.u_plus_e[e];
      if (up > 0.0) bloss += up / dx;
    } else {
      const double ue = g.u_e[e];
      if (ue >= 0.0) bloss += ue / dx;
    }
  }
  // ---- y faces ----
  if (j > 0) {  // south face: this cell is R (north)
    const int64_t L = cell - nx;
    const double dxs = dx_at(g.lat[j - 1]);
    double rl, rr;
    face_rates(g.kxxyy[L], g.kxxyy[cell], g.kmv ? g.kmv[cell] : 0.0, split, g.v[cell], VP(cell),
               VM(cell), dy, rl, rr);
    const double dPL = g.dP[L];
    const bool ok = dPL > 0.0 && dPc > 0.0;
    const double dxf = 0.5 * (dxs + dx);
    const double trR = ok ? (dxf / dx) * (0.5 * (dPL + dPc) / dPc) : 1.0;
    diag += rr * trR;
    oS = -(rl * trR);
  } else {
    const double latf = g.lat[0] - g.dlat / 2.0;
    const double tr = dx_at(latf) / dx;
    const double vm = VM(cell);
    if (vm > 0.0) bloss += vm / dy * tr;
  }
  if (j < ny - 1) {  // north face: this cell is L (south)
    const int64_t R = cell + nx;
    const double dxn = dx_at(g.lat[j + 1]);
    double rl, rr;
    face_rates(g.kxxyy[cell], g.kxxyy[R], g.kmv ? g.kmv[R] : 0.0, split, g.v[R], VP(R), VM(R), dy,
               rl, rr);
    const double dPR = g.dP[R];
    const bool ok = dPc > 0.0 && dPR > 0.0;
    const double dxf = 0.5 * (dx + dxn);
    const double trL = ok ? (dxf / dx) * (0.5 * (dPc + dPR) / dPc) : 1.0;
    diag += rl * trL;
    oN = -(rr * trL);
  } else {
    const double latf = g.lat[ny - 1] + g.dlat / 2.0;
    const double tr = dx_at(latf) / dx;
    const int64_t e = (int64_t)k * nx + i;
    if (split) {
      const double vp = g.v_plus_n[e];
      if (vp > 0.0) bloss += vp / dy * tr;
    } else {
      const double vn = g.v_n[e];
      if (vn >= 0.0) bloss += vn / dy * tr;
    }
  }
  if (lat_loss) {
    lat_loss[cell] = bloss;
    if (!Tst) return;
  }
  diag += bloss;
  // ---- vertical advection (interface k = bottom face, k+1 = top face) ----
  if (dPc > 0.0) {
    if (k >= 1) {
      const double wd = g.w_plus[cell], wu = g.w_minus[cell];
      if (wd > 0.0) diag += wd / dPc;
      if (wu > 0.0) oB += -wu / dPc;
    }
    const double wd1 = g.w_plus[cell + nxy], wu1 = g.w_minus[cell + nxy];
    if (k < nz - 1 && wd1 > 0.0) oT += -wd1 / dPc;
    if (wu1 > 0.0) diag += wu1 / dPc;
  }
  // ---- vertical diffusion ----
  const double Dzc = g.Dz[cell];
  const double rhoc = (Dzc > 0.0 && dPc > 0.0) ? dPc / (kGravity * Dzc) : 0.0;
  if (k < nz - 1) {  // interface (k, k+1): this cell is the lower layer
    const int64_t U = cell + nxy;
    const double Dzu = g.Dz[U];
    if (Dzc > 0.0 && Dzu > 0.0) {
      const double Kc = g.kzz[cell], Ku = g.kzz[U];
      const double Kf = 2.0 * Kc * Ku / (Kc + Ku + 1e-30);
      const double dist = 0.5 * (Dzc + Dzu);
      const double dPu = g.dP[U];
      const double rhou = (Dzu > 0.0 && dPu > 0.0) ? dPu / (kGravity * Dzu) : 0.0;
      const double rf = 0.5 * (rhoc + rhou);
      const bool both = rhoc > 0.0 && rhou > 0.0;
      const double ratio = both ? rf / (rhoc > 0.0 ? rhoc : 1.0) : 1.0;
      const double c0 = Kf / (Dzc * dist) * ratio;
      oT += -c0;
      diag += c0;
    }
  }
  if (k > 0) {  // interface (k-1, k): this cell is the upper layer
    const int64_t Lw = cell - nxy;
    const double Dzl = g.Dz[Lw];
    if (Dzl > 0.0 && Dzc > 0.0) {
      const double Kl = g.kzz[Lw], Kc = g.kzz[cell];
      const double Kf = 2.0 * Kl * Kc / (Kl + Kc + 1e-30);
      const double dist = 0.5 * (Dzl + Dzc);
      const double dPl = g.dP[Lw];
      const double rhol = (Dzl > 0.0 && dPl > 0.0) ? dPl / (kGravity * Dzl) : 0.0;
      const double rf = 0.5 * (rhol + rhoc);
      const bool both = rhol > 0.0 && rhoc > 0.0;
      const double ratio = both ? rf / (rhoc > 0.0 ? rhoc : 1.0) : 1.0;
      const double c1 = Kf / (Dzc * dist) * ratio;
      oB += -c1;
      diag += c1;
    }
  }
  // ---- convective mass flux ----
  if (g.cmfmc) {
    const bool okc = Dzc > 0.0 && dPc > 0.0;
    const double sDz = Dzc > 0.0 ? Dzc : 1.0;
    const double rc = dPc / (kGravity * sDz);
    const double srho = rc > 0.0 ? rc : 1.0;
    const double Ft = fmax(g.cmfmc[cell + nxy], 0.0);  // top interface of k
    if (okc && Ft > 0.0) {
      const double src = Ft / (srho * sDz);
      diag += src;
      if (k < nz - 1) {
        const double Dzu = g.Dz[cell + nxy], dPu = g.dP[cell + nxy];
        if (Dzu > 0.0 && dPu > 0.0) oT += -src;
      }
    }
    if (k >= 1) {
      const double Fb = fmax(g.cmfmc[cell], 0.0);  // bottom interface of k
      const double Dzl = g.Dz[cell - nxy], dPl = g.dP[cell - nxy];
      const bool okl = Dzl > 0.0 && dPl > 0.0;
      if (okl && Fb > 0.0 && okc) {
        const double rec = Fb / (srho * sDz);
        oB += -rec;
        diag += rec;
      }
    }
  }
  if (rowsum) rowsum[cell] = diag + oW + oE + oS + oN + oB + oT;
  // ---- concentration form: off(c, nb) *= rho_c / rho_nb (pressure-form
  // grids keep the block as assembled, operator.py:341) ----
  const double rc = rho_of(dPc, Dzc);
  auto sim = [&](double v, int64_t nb) {
    return (v == 0.0 || g.pressure_form) ? v : rc * v / rho_of(g.dP[nb], g.Dz[nb]);
  };
  Tst[0 * NN + cell] = diag;
  Tst[1 * NN + cell] = i > 0 ? sim(oW, cell - 1) : px ? sim(oW, cell + nx - 1) : 0.0;
  Tst[2 * NN + cell] = i < nx - 1 ? sim(oE, cell + 1) : px ? sim(oE, cell - (nx - 1)) : 0.0;
  Tst[3 * NN + cell] = j > 0 ? sim(oS, cell - nx) : 0.0;
  Tst[4 * NN + cell] = j < ny - 1 ? sim(oN, cell + nx) : 0.0;
  Tst[5 * NN + cell] = k > 0 ? sim(oB, cell - nxy) : 0.0;
  Tst[6 * NN + cell] = k < nz - 1 ? sim(oT, cell + nxy) : 0.0;
}

// |row sum| per day of laterally interior cells; rows of the concentration
// form weighted by rho reduce to the pressure-form row sums.
__global__ void k_mass_rows(int nz, int ny, int nx, const double* const* Tst, const double* const* rho,
                            double* out_int, double* out_top) {
  const int b = blockIdx.y;
  const int64_t NN = (int64_t)nz * ny * nx;
  const double* T = Tst[b];
  const double* w = rho[b];
  const int iy = ny - 2, ix = nx - 2;
  const int64_t per = (int64_t)nz * iy * ix;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < per;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(e % ix);
    const int j = 1 + (int)((e / ix) % iy);
    const int k = (int)(e / ((int64_t)ix * iy));
    const int64_t c = ((int64_t)k * ny + j) * nx + i;
    const int64_t nxy = (int64_t)nx * ny;
    double r = T[c] * w[c];
    r += T[NN + c] * w[c - 1];
    r += T[2 * NN + c] * w[c + 1];
    r += T[3 * NN + c] * w[c - nx];
    r += T[4 * NN + c] * w[c + nx];
    if (k > 0) r += T[5 * NN + c] * w[c - nxy];
    if (k < nz - 1) r += T[6 * NN + c] * w[c + nxy];
    const double v = fabs(r / w[c] * 86400.0);
    const int64_t q = ((int64_t)(j - 1)) * ix + (i - 1);
    if (k < nz - 1)
      out_int[(int64_t)b * (nz - 1) * iy * ix + (int64_t)k * iy * ix + q] = v;
    else
      out_top[(int64_t)b * iy * ix + q] = v;
  }
}

// y_v = beta y_v + alpha S_v x_v (or S_v^T x_v) for 7-point stencils S_v
// ([7][N]: centre, W, E, S, N, below, above; entries pointing outside the
// grid are ignored) and vectors x_v, one (vector, cell) per thread.
__global__ void k_stencil_apply(int nz, int ny, int nx, int px, const double* __restrict__ S_all,
                                const double* __restrict__ x_all, double alpha, double beta, int trans,
                                double* __restrict__ y_all) {
  const int64_t N = (int64_t)nz * ny * nx;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const double* S = S_all + (int64_t)blockIdx.y * 7 * N;
  const double* x = x_all + (int64_t)blockIdx.y * N;
  double* y = y_all + (int64_t)blockIdx.y * N;
  int64_t nb[6];
  bool has[6];
  stencil_nbrs(p, nz, ny, nx, px, nb, has);
  double acc = S[p] * x[p];
  if (!trans) {
#pragma unroll
    for (int d = 0; d < 6; ++d)
      if (has[d]) acc += S[(d + 1) * N + p] * x[nb[d]];
  } else {
    // (S^T x)_p = sum over the neighbours q of their entries pointing at p
    // (the opposite direction: W <-> E, S <-> N, B <-> T)
    const int opp[6] = {2, 1, 4, 3, 6, 5};
#pragma unroll
    for (int d = 0; d < 6; ++d)
      if (has[d]) acc += S[opp[d] * N + nb[d]] * x[nb[d]];
  }
  y[p] = (beta != 0.0 ? beta * y[p] : 0.0) + alpha * acc;
}

}  // namespace

int stencil_apply(int nz, int ny, int nx, int px, int n_vec, const double* S, const double* x, double alpha,
                  double beta, int trans, double* y, cudaStream_t st) {
  const int64_t N = (int64_t)nz * ny * nx;
  dim3 g((unsigned)((N + 255) / 256), n_vec);
  k_stencil_apply<<<g, 256, 0, st>>>(nz, ny, nx, px, S, x, alpha, beta, trans, y);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

int assemble_transport(int nz, int ny, int nx, const orbit_met_t* met, double* T, double* rowsum,
                       double* lat_loss, cudaStream_t st) {
  const int64_t NN = (int64_t)nz * ny * nx;
  const int threads = 128;
  k_assemble<<<(unsigned)((NN + threads - 1) / threads), threads, 0, st>>>(nz, ny, nx, *met, T, rowsum, lat_loss);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

int mass_balance_rows(int nz, int ny, int nx, int nbins, const double* const* Tst,
                      const double* const* rho, double* out_int, double* out_top, cudaStream_t st) {
  const int64_t per = (int64_t)nz * (ny - 2) * (nx - 2);
  dim3 g((unsigned)((per + 255) / 256), nbins);
  k_mass_rows<<<g, 256, 0, st>>>(nz, ny, nx, Tst, rho, out_int, out_top);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

}  // namespace orbit
