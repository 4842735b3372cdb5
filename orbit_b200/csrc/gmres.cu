// K5: batched periodic-orbit GMRES on the device, forward and transposed.
//
// Mirrors solve_orbit_one_species (orbit/core/orbit.py:123-210) and
// solve_orbit_adjoint_one_species (orbit/core/orbit_adjoint.py:70-144) with
// the restarted GMRES of scipy.sparse.linalg.gmres as they call it
// (restart 30, atol = tol ||s||, x0 = warm start or s, one true residual per
// cycle).  Many orbits advance in lockstep; each leaves the active set when its
// own residual estimate reaches its own tolerance.  Orthogonalisation is
// classical Gram-Schmidt with one reorthogonalisation (CGS2), the Hessenberg
// column, Givens rotations and the least-squares update stay FP64 on the
// device; the host only reads the per-orbit residual estimates to steer.
//
// With FP32 factors the monodromy M~ used inside GMRES is inexact; the orbit is
// then obtained by FP64 iterative refinement of the monodromy residual: the
// residual s - (I - M) c uses FP64-refined bin solves (one FP32 re-solve of the
// FP64 stencil residual per bin), and the correction solves (I - M~) d = r.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "handles.h"

namespace orbit {

int launch_chain(orbit_factor_s* f, int B, const int* d_orbit_ids, int trans, int tau0, int tau1,
                 const double* E, double escale, cudaStream_t st);
int launch_chain_x(orbit_factor_s* f, double* X, int B, const int* d_orbit_ids, int trans, int tau0,
                   int tau1, const double* E, double escale, cudaStream_t st);

namespace {

constexpr int kRedBlocks = 48;
constexpr int kVT = 256;

__global__ void k_perm_gather(double* dst, int64_t dstride, const double* src, int64_t sstride, int nvec,
                              const int32_t* perm, const int* ids, int64_t N) {
  const int o = ids[blockIdx.y];
  for (int v = 0; v < nvec; ++v) {
    double* d = dst + (int64_t)o * dstride + (int64_t)v * N;
    const double* s = src + (int64_t)o * sstride + (int64_t)v * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
      d[p] = s[perm[p]];
  }
}

__global__ void k_perm_scatter(double* dst, int64_t dstride, const double* src, int64_t sstride, int nvec,
                               const int32_t* perm, const int* ids, int64_t N) {
  const int o = ids[blockIdx.y];
  for (int v = 0; v < nvec; ++v) {
    double* d = dst + (int64_t)o * dstride + (int64_t)v * N;
    const double* s = src + (int64_t)o * sstride + (int64_t)v * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
      d[perm[p]] = s[p];
  }
}

// dst = a*x + b*y ; scalars from device arrays (per orbit, index o*ld+off) or constants
struct Scal {
  const double* p;
  int ld, off;
  double c;
  __device__ double get(int o) const { return p ? p[o * ld + off] * c : c; }
};

__global__ void k_lincomb(double* dst, int64_t ds, Scal a, const double* x, int64_t xs, Scal b,
                          const double* y, int64_t ys, const int* ids, int64_t N) {
  const int o = ids[blockIdx.y];
  const double av = a.get(o), bv = b.get(o);
  double* d = dst + (int64_t)o * ds;
  const double* xv = x ? x + (int64_t)o * xs : nullptr;
  const double* yv = y ? y + (int64_t)o * ys : nullptr;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (xv) v += av * xv[p];
    if (yv) v += bv * yv[p];
    d[p] = v;
  }
}

// partial[o][i][blk] = sum_p X_i[p] * y[p], X_i = X + o*xs + i*N
__global__ void k_multidot(double* partial, const double* X, int64_t xs, int nvec, const double* y,
                           int64_t ys, const int* ids, int64_t N) {
  __shared__ double red[kVT / 32][32];
  const int o = ids[blockIdx.y];
  const double* yv = y + (int64_t)o * ys;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = 0; i0 < nvec; i0 += 32) {
    const int ni = min(32, nvec - i0);
    double acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
      const double yy = yv[p];
#pragma unroll
      for (int q = 0; q < 32; ++q)
        if (q < ni) acc[q] = fma(X[(int64_t)o * xs + (int64_t)(i0 + q) * N + p], yy, acc[q]);
    }
    for (int q = 0; q < ni; ++q) {
      double v = warp_sum(acc[q]);
      if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < ni) {
      double sum = 0.0;
      for (int w = 0; w < kVT / 32; ++w) sum += red[w][threadIdx.x];
      partial[((int64_t)o * 32 * 33 + (i0 + threadIdx.x)) * kRedBlocks + blockIdx.x] = sum;
    }
    __syncthreads();
  }
}

// out[o*ld + off + i] = (accumulate ? out : 0) + sum_blk partial
__global__ void k_reduce_partials(double* out, int ld, int off, const double* partial, int nvec,
                                  const int* ids, int accumulate) {
  const int o = ids[blockIdx.x];
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < kRedBlocks; ++b) s += partial[((int64_t)o * 32 * 33 + i) * kRedBlocks + b];
    out[o * ld + off + i] = accumulate ? out[o * ld + off + i] + s : s;
  }
}

// w -= sum_i h[o*ld+off+i] * V_i   (sign = -1)   or  x += sum_i y_i V_i (sign = +1)
__global__ void k_combine(double* w, int64_t ws, const double* V, int64_t vs, const double* h, int ld,
                          int off, const int* ncol_dev, int ncol_const, double sign, const int* ids,
                          int64_t N) {
  const int o = ids[blockIdx.y];
  const int nc = ncol_dev ? ncol_dev[o] : ncol_const;
  double* wv = w + (int64_t)o * ws;
  const double* hv = h + o * ld + off;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int i = 0; i < nc; ++i) acc = fma(hv[i], V[(int64_t)o * vs + (int64_t)i * N + p], acc);
    wv[p] += sign * acc;
  }
}

// scal layout per orbit (ld kScal): see indices below
constexpr int kScal = 16;
enum { S_NORM = 0, S_H0 = 1, S_PRES = 2, S_BREAK = 3, S_TMP = 4, S_SN = 5, S_NEG = 6 };

// v = w / ||w||, record breakdown.  hcol points to H column col (ld R+1).
__global__ void k_normalize(double* Vnext, const double* w, int64_t vs, int64_t ws, double* H, int hld,
                            int col, double* scal, const int* ids, int64_t N) {
  const int o = ids[blockIdx.y];
  const double hn = sqrt(fmax(scal[o * kScal + S_NORM], 0.0));
  const double h0 = sqrt(fmax(scal[o * kScal + S_H0], 0.0));
  const bool brk = hn <= 2.220446049250313e-16 * h0;
  double* v = Vnext + (int64_t)o * vs;
  const double* wv = w + (int64_t)o * ws;
  const double inv = brk ? 0.0 : 1.0 / hn;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
    v[p] = brk ? wv[p] : wv[p] * inv;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    H[(int64_t)o * hld * 32 + (int64_t)col * hld + col + 1] = brk ? 0.0 : hn;
    scal[o * kScal + S_BREAK] = brk ? 1.0 : 0.0;
  }
}

// Apply previous rotations to column col, build the new one, update g.
__global__ void k_givens(double* H, int hld, double* cs, double* sn, double* g, int col, double* scal,
                         const int* ids, int B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B) return;
  const int o = ids[t];
  double* h = H + (int64_t)o * hld * 32 + (int64_t)col * hld;
  double* c = cs + o * 32;
  double* s = sn + o * 32;
  double* gg = g + o * 33;
  for (int k = 0; k < col; ++k) {
    const double n0 = h[k], n1 = h[k + 1];
    h[k] = c[k] * n0 + s[k] * n1;
    h[k + 1] = -s[k] * n0 + c[k] * n1;
  }
  const double a = h[col], b = h[col + 1];
  double cc, ss, r;
  if (b == 0.0) {
    cc = 1.0; ss = 0.0; r = a;
  } else if (a == 0.0) {
    cc = 0.0; ss = 1.0; r = b;
  } else {
    r = hypot(a, b);
    cc = a / r;
    ss = b / r;
  }
  c[col] = cc;
  s[col] = ss;
  h[col] = r;
  h[col + 1] = 0.0;
  const double tmp = -ss * gg[col];
  gg[col] = cc * gg[col];
  gg[col + 1] = tmp;
  scal[o * kScal + S_PRES] = fabs(tmp);
}

// y = H(0:nc,0:nc)^-1 g(0:nc) by back substitution, stored in g's slot ysl
__global__ void k_ysolve(const double* H, int hld, const double* g, double* y, const int* ncol,
                         const int* ids, int B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B) return;
  const int o = ids[t];
  const int nc = ncol[o];
  if (nc <= 0) return;
  const double* h = H + (int64_t)o * hld * 32;
  double* yy = y + o * 33;
  for (int i = 0; i < nc; ++i) yy[i] = g[o * 33 + i];
  if (h[(int64_t)(nc - 1) * hld + nc - 1] == 0.0) yy[nc - 1] = 0.0;
  for (int k = nc - 1; k > 0; --k) {
    if (yy[k] != 0.0) {
      yy[k] /= h[(int64_t)k * hld + k];
      const double tmp = yy[k];
      for (int i = 0; i < k; ++i) yy[i] -= tmp * h[(int64_t)k * hld + i];
    }
  }
  if (yy[0] != 0.0) yy[0] /= h[0];
}

// v = v / sqrt(scal[slot])
__global__ void k_scale_inv_norm(double* v, int64_t vs, const double* scal, int slot, const int* ids,
                                 int64_t N) {
  const int o = ids[blockIdx.y];
  const double nrm = sqrt(fmax(scal[o * kScal + slot], 0.0));
  const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
  double* vv = v + (int64_t)o * vs;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
    vv[p] *= inv;
}

__global__ void k_init_g(double* g, double* scal, const int* ids, int B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B) return;
  const int o = ids[t];
  for (int i = 0; i < 33; ++i) g[o * 33 + i] = 0.0;
  g[o * 33] = sqrt(fmax(scal[o * kScal + S_NORM], 0.0));
}

// r = b - A x on the permuted 7-point stencil (FP64), trans: r = b - A^T x
__global__ void k_stencil_resid(double* r, int64_t rs, const double* b, int64_t bs, const double* x,
                                int64_t xs, const double* Ast, int tau, const int32_t* perm,
                                const int32_t* iperm, int nz, int ny, int nx, int px, int trans, const int* ids,
                                const int* set_of, int n_bins) {
  const int o = ids[blockIdx.y];
  const int64_t N = (int64_t)nz * ny * nx;
  const double* A = Ast + ((int64_t)set_of[o] * n_bins + tau) * 7 * N;
  const double* xv = x + (int64_t)o * xs;
  const double* bv = b + (int64_t)o * bs;
  double* rv = r + (int64_t)o * rs;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = perm[p];
    double acc = A[c] * xv[p];
    // neighbours: W E S N B T, opposite directions E W N S T B
    int64_t nb[6];
    bool has[6];
    stencil_nbrs(c, nz, ny, nx, px, nb, has);
    const int opp[6] = {2, 1, 4, 3, 6, 5};
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      if (!has[d]) continue;
      const double a = trans ? A[(int64_t)opp[d] * N + nb[d]] : A[(int64_t)(d + 1) * N + c];
      acc = fma(a, xv[iperm[nb[d]]], acc);
    }
    rv[p] = bv[p] - acc;
  }
}

// Block-cyclic residual of the eight bin equations A_tau c_{tau+1} = c_tau + fs e_tau
// (c_0 := c_8):  R_tau = fs e_tau + c_tau - A_tau c_{tau+1}, FP64, permuted order.
// C: per orbit 9 vectors (slot 0 unused, c_0 read from slot 8); E, R: per orbit 8 vectors.
__global__ void k_block_resid(double* R, const double* E, double fs, const double* Cb, const double* Ast,
                              const int32_t* perm, const int32_t* iperm, int nz, int ny, int nx, int px,
                              const int* ids, const int* set_of) {
  const int o = ids[blockIdx.y];
  const int64_t N = (int64_t)nz * ny * nx;
  const double* C = Cb + (int64_t)o * 9 * N;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = perm[p];
    int64_t nb[6];
    bool has[6];
    stencil_nbrs(c, nz, ny, nx, px, nb, has);
    int64_t q[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) q[d] = has[d] ? iperm[nb[d]] : 0;
    for (int tau = 0; tau < 8; ++tau) {
      const double* A = Ast + ((int64_t)set_of[o] * 8 + tau) * 7 * N;
      const double* cin = C + (int64_t)(tau == 0 ? 8 : tau) * N;
      const double* cout = C + (int64_t)(tau + 1) * N;
      double acc = A[c] * cout[p];
#pragma unroll
      for (int d = 0; d < 6; ++d)
        if (has[d]) acc = fma(A[(int64_t)(d + 1) * N + c], cout[q[d]], acc);
      const double rhs = cin[p] + (E ? fs * E[((int64_t)o * 8 + tau) * N + p] : 0.0);
      R[((int64_t)o * 8 + tau) * N + p] = rhs - acc;
    }
  }
}

// Block-cyclic residual of the eight transposed bin equations
// A_tau^T (lam_tau - R_tau) = lam_{tau+1} (lam_8 := lam_0), FP64, permuted
// order: rho_tau = lam_{tau+1} - A_tau^T (lam_tau - R_tau).  Written in the
// forcing layout of the transposed chain, which adds E[tau+1] before P_tau^T:
// Rs[k] = rho_{k-1} for k = 1..7, Rs[0] = 0, and rho_7 (the input of the last
// bin) into rho7.  L: per orbit 9 vectors (lam_0..lam_7 in slots 0..7);
// R: per orbit 8 receptors.
__global__ void k_block_resid_T(double* Rs, double* rho7, int64_t r7s, const double* R, const double* Lb,
                                const double* Ast, const int32_t* perm, const int32_t* iperm, int nz, int ny,
                                int nx, int px, const int* ids, const int* set_of) {
  const int o = ids[blockIdx.y];
  const int64_t N = (int64_t)nz * ny * nx;
  const double* L = Lb + (int64_t)o * 9 * N;
  const double* Ro = R + (int64_t)o * 8 * N;
  double* Ro_s = Rs + (int64_t)o * 8 * N;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = perm[p];
    int64_t nb[6];
    bool has[6];
    stencil_nbrs(c, nz, ny, nx, px, nb, has);
    const int opp[6] = {2, 1, 4, 3, 6, 5};
    int64_t q[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) q[d] = has[d] ? iperm[nb[d]] : 0;
    Ro_s[p] = 0.0;
    for (int tau = 0; tau < 8; ++tau) {
      const double* A = Ast + ((int64_t)set_of[o] * 8 + tau) * 7 * N;
      const double* lam = L + (int64_t)tau * N;
      const double* rr = Ro + (int64_t)tau * N;
      // (A^T mu)_p = A_pp mu_p + sum over neighbours q of A_qp mu_q, mu = lam - R
      double acc = A[c] * (lam[p] - rr[p]);
#pragma unroll
      for (int d = 0; d < 6; ++d)
        if (has[d]) acc = fma(A[(int64_t)opp[d] * N + nb[d]], lam[q[d]] - rr[q[d]], acc);
      const double rho = L[(int64_t)((tau + 1) & 7) * N + p] - acc;
      if (tau < 7) Ro_s[(int64_t)(tau + 1) * N + p] = rho;
      else rho7[(int64_t)o * r7s + p] = rho;
    }
  }
}

__global__ void k_count_neg(double* partial, const double* X, int64_t xs, int64_t len, const int* ids) {
  __shared__ double red[kVT / 32];
  const int o = ids[blockIdx.y];
  const double* xv = X + (int64_t)o * xs;
  double c = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < len; p += (int64_t)gridDim.x * blockDim.x)
    c += xv[p] < 0.0 ? 1.0 : 0.0;
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kVT / 32; ++w) s += red[w];
    partial[((int64_t)o * 32 * 33) * kRedBlocks + blockIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
struct Ctx {
  orbit_factor_s* f;
  cudaStream_t st;
  int64_t N;
  int R;       // restart
  int hld;     // R + 1
  bool mixed;
  int trans;
  double* Sv;  // per orbit N: s
  double* Xv;  // per orbit N: iterate
  double* Rv;  // per orbit N: residual / work
  double* Dv;  // per orbit N: correction
  double* Tv;  // per orbit N: scratch
  double* XS;  // per orbit 9N: IR scratch chain buffer
  double* partial;
  int64_t vs;  // per-orbit stride of the N-vectors (N)
};

inline dim3 vgrid(int64_t N, int B) {
  int64_t bx = (N + kVT - 1) / kVT;
  if (bx > 1024) bx = 1024;
  return dim3((unsigned)bx, (unsigned)B);
}

int upload_ids(Ctx& c, const std::vector<int>& ids, int* d_ids) {
  ORBIT_CUDA_TRY(cudaMemcpyAsync(d_ids, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice, c.st));
  return ORBIT_OK;
}

// squared norms into scal[S_NORM] (or another slot)
int sqnorm(Ctx& c, const double* v, int64_t vstride, const int* d_ids, int B, int slot) {
  orbit_factor_s* f = c.f;
  k_multidot<<<dim3(kRedBlocks, B), kVT, 0, c.st>>>(c.partial, v, vstride, 1, v, vstride, d_ids, c.N);
  note_launch();
  k_reduce_partials<<<B, 32, 0, c.st>>>(f->scal, kScal, slot, c.partial, 1, d_ids, 0);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

int fetch_scal(Ctx& c) {
  orbit_factor_s* f = c.f;
  ORBIT_CUDA_TRY(cudaMemcpyAsync(f->h_scal, f->scal, sizeof(double) * kScal * f->n_orbits,
                                 cudaMemcpyDeviceToHost, c.st));
  ORBIT_CUDA_TRY(cudaMemcpyAsync(f->h_status, f->status, sizeof(int), cudaMemcpyDeviceToHost, c.st));
  ORBIT_CUDA_TRY(cudaStreamSynchronize(c.st));
  if (*f->h_status != 0) {
    int code = *f->h_status;
    set_last_error(code == ORBIT_ERR_TIMEOUT ? "device spin-wait timed out"
                   : code == ORBIT_ERR_PIVOT ? "zero or non-finite pivot in the numeric factorization"
                                             : "device status error");
    return code;
  }
  return ORBIT_OK;
}

// One bin with FP64 iterative refinement (FP32 factors): X[tau+1] = P_tau (X[tau] + fscale E[tau]).
// Forward only here; the transposed variant mirrors it.
int refined_bin(Ctx& c, const int* d_ids, int B, int tau, int tau1, const double* E, double fscale) {
  orbit_factor_s* f = c.f;
  orbit_symbolic_s* sy = f->sym;
  const int64_t N = c.N;
  const int64_t xs = 9 * N;
  double* X = f->X;
  double* XS = c.XS;
  const dim3 g = vgrid(N, B);
  const int trans = c.trans;
  // input b of this bin (forward: X[tau] + fscale E[tau]; transposed: X[tau+1] + fscale E[tau+1] unless last)
  const int bin_in = trans ? tau + 1 : tau;
  const int bin_out = trans ? tau : tau + 1;
  const double* Ein = nullptr;
  if (E) {
    if (!trans) Ein = E + (int64_t)tau * N;
    else if (tau + 1 < tau1) Ein = E + (int64_t)(tau + 1) * N;
  }
  Scal one{nullptr, 0, 0, 1.0}, fs{nullptr, 0, 0, fscale};
  // XS[bin_in] = b
  k_lincomb<<<g, kVT, 0, c.st>>>(XS + bin_in * N, xs, one, X + bin_in * N, xs, fs, Ein, 8 * N, d_ids, N);
  note_launch();
  int rc = launch_chain_x(f, XS, B, d_ids, trans, tau, tau + 1, nullptr, 0.0, c.st);
  if (rc) return rc;
  // xhat -> Tv ; r = b - A xhat -> XS[bin_in]
  k_lincomb<<<g, kVT, 0, c.st>>>(c.Tv, c.vs, one, XS + bin_out * N, xs, one, nullptr, 0, d_ids, N);
  note_launch();
  k_stencil_resid<<<g, kVT, 0, c.st>>>(c.Rv, c.vs, XS + bin_in * N, xs, c.Tv, c.vs, f->A_stencil, tau,
                                       sy->d.perm, sy->d.iperm, sy->S.nz, sy->S.ny, sy->S.nx, sy->S.periodic_x, trans, d_ids,
                                       f->set_of, f->n_bins);
  note_launch();
  k_lincomb<<<g, kVT, 0, c.st>>>(XS + bin_in * N, xs, one, c.Rv, c.vs, one, nullptr, 0, d_ids, N);
  note_launch();
  rc = launch_chain_x(f, XS, B, d_ids, trans, tau, tau + 1, nullptr, 0.0, c.st);
  if (rc) return rc;
  // X[bin_out] = xhat + correction
  k_lincomb<<<g, kVT, 0, c.st>>>(X + bin_out * N, xs, one, c.Tv, c.vs, one, XS + bin_out * N, xs, d_ids, N);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

// Full chain on f->X (accurate): forward reads X[0] writes X[1..8]; transposed reads X[8] writes X[7..0].
int chain_accurate(Ctx& c, const int* d_ids, int B, const double* E, double fscale, int tau0 = 0,
                   int tau1 = 8) {
  orbit_factor_s* f = c.f;
  if (!c.mixed) return launch_chain(f, B, d_ids, c.trans, tau0, tau1, E, fscale, c.st);
  if (!c.trans) {
    for (int t = tau0; t < tau1; ++t) {
      int rc = refined_bin(c, d_ids, B, t, tau1, E, fscale);
      if (rc) return rc;
    }
  } else {
    for (int t = tau1 - 1; t >= tau0; --t) {
      int rc = refined_bin(c, d_ids, B, t, tau1, E, fscale);
      if (rc) return rc;
    }
    if (E) {
      // transposed chain adds the forcing after the last bin
      const dim3 g = vgrid(c.N, B);
      Scal one{nullptr, 0, 0, 1.0}, fs{nullptr, 0, 0, fscale};
      k_lincomb<<<g, kVT, 0, c.st>>>(f->X + (int64_t)tau0 * c.N, 9 * c.N, one, f->X + (int64_t)tau0 * c.N,
                                     9 * c.N, fs, E + (int64_t)tau0 * c.N, 8 * c.N, d_ids, c.N);
      note_launch();
    }
  }
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

// w = v - M v  (inexact = FP32 chain in mixed mode, exact chain in FP64 mode, accurate = refined)
int matvec(Ctx& c, const double* v, int64_t vstride, double* w, int64_t wstride, const int* d_ids, int B,
           bool accurate) {
  orbit_factor_s* f = c.f;
  const int64_t N = c.N;
  const dim3 g = vgrid(N, B);
  Scal one{nullptr, 0, 0, 1.0}, mone{nullptr, 0, 0, -1.0};
  const int in = c.trans ? 8 : 0, out = c.trans ? 0 : 8;
  k_lincomb<<<g, kVT, 0, c.st>>>(f->X + in * N, 9 * N, one, v, vstride, one, nullptr, 0, d_ids, N);
  note_launch();
  int rc = (accurate && c.mixed) ? chain_accurate(c, d_ids, B, nullptr, 0.0)
                                 : launch_chain(f, B, d_ids, c.trans, 0, 8, nullptr, 0.0, c.st);
  if (rc) return rc;
  k_lincomb<<<g, kVT, 0, c.st>>>(w, wstride, one, v, vstride, mone, f->X + out * N, 9 * N, d_ids, N);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

// Restarted GMRES on (I - M) x = b for the orbits in `act`; x, b per orbit (stride vs).
// atol per orbit; iters accumulated; converged flags set.  rn_out gets the final true residual norm.
int gmres(Ctx& c, std::vector<int> act, double* b, double* x, const std::vector<double>& atol,
          int maxiter, bool accurate_mv, std::vector<int>& iters, std::vector<int>& conv,
          std::vector<double>& rn_out, std::vector<int>& matvecs, bool x_is_zero,
          bool trust_estimate = false) {
  orbit_factor_s* f = c.f;
  const int64_t N = c.N;
  const int R = c.R;
  const int hld = c.hld;
  int* d_ids = f->orbit_ids;
  std::vector<int> ncol_h(f->n_orbits, 0);
  int* d_ncol = f->task_counter + 1;  // small int scratch after the task counter
  Scal one{nullptr, 0, 0, 1.0}, mone{nullptr, 0, 0, -1.0};
  auto V_of = [&](int i) { return f->V + (int64_t)i * N; };
  const int64_t vstr = (int64_t)(R + 1) * N;
  // initial residual r = b - A x  -> V0 (unnormalised)
  int rc = upload_ids(c, act, d_ids);
  if (rc) return rc;
  int B = (int)act.size();
  if (B == 0) return ORBIT_OK;
  if (x_is_zero) {
    k_lincomb<<<vgrid(N, B), kVT, 0, c.st>>>(V_of(0), vstr, one, b, c.vs, one, nullptr, 0, d_ids, N);
    note_launch();
  } else {
    rc = matvec(c, x, c.vs, c.Rv, c.vs, d_ids, B, accurate_mv);
    if (rc) return rc;
    for (int o : act) matvecs[o]++;
    k_lincomb<<<vgrid(N, B), kVT, 0, c.st>>>(V_of(0), vstr, one, b, c.vs, mone, c.Rv, c.vs, d_ids, N);
    note_launch();
  }
  rc = sqnorm(c, V_of(0), vstr, d_ids, B, S_NORM);
  if (rc) return rc;
  rc = fetch_scal(c);
  if (rc) return rc;
  {
    std::vector<int> keep;
    for (int o : act) {
      double rn = std::sqrt(std::max(f->h_scal[o * kScal + S_NORM], 0.0));
      rn_out[o] = rn;
      if (rn < atol[o]) conv[o] = 1;
      else keep.push_back(o);
    }
    act.swap(keep);
  }
  for (int cycle = 0; cycle < maxiter && !act.empty(); ++cycle) {
    B = (int)act.size();
    rc = upload_ids(c, act, d_ids);
    if (rc) return rc;
    // V0 = r / ||r|| ; g = [||r||, 0, ...]
    k_init_g<<<(B + 63) / 64, 64, 0, c.st>>>(f->gv, f->scal, d_ids, B);
    note_launch();
    k_scale_inv_norm<<<vgrid(N, B), kVT, 0, c.st>>>(V_of(0), vstr, f->scal, S_NORM, d_ids, N);
    note_launch();
    std::vector<int> inner = act;
    std::vector<char> est_done(f->n_orbits, 0);
    std::vector<double> pres_h(f->n_orbits, 0.0);
    for (int o : act) ncol_h[o] = 0;
    for (int col = 0; col < R && !inner.empty(); ++col) {
      const int Bi = (int)inner.size();
      rc = upload_ids(c, inner, d_ids);
      if (rc) return rc;
      const dim3 g = vgrid(N, Bi);
      // w = A v_col -> Rv
      rc = matvec(c, V_of(col), vstr, c.Rv, c.vs, d_ids, Bi, accurate_mv);
      if (rc) return rc;
      for (int o : inner) matvecs[o]++;
      // h0 = ||w||^2
      rc = sqnorm(c, c.Rv, c.vs, d_ids, Bi, S_H0);
      if (rc) return rc;
      // CGS2
      for (int pass = 0; pass < 2; ++pass) {
        k_multidot<<<dim3(kRedBlocks, Bi), kVT, 0, c.st>>>(c.partial, f->V, vstr, col + 1, c.Rv, c.vs, d_ids, N);
        note_launch();
        k_reduce_partials<<<Bi, 32, 0, c.st>>>(f->Hd, hld * 32, col * hld, c.partial, col + 1, d_ids, pass);
        note_launch();
        // w -= V h (pass 0 uses the full h; pass 1 must use only the increment) -> use Tv copy of increment
        if (pass == 0) {
          k_combine<<<g, kVT, 0, c.st>>>(c.Rv, c.vs, f->V, vstr, f->Hd, hld * 32, col * hld, nullptr, col + 1,
                                         -1.0, d_ids, N);
          note_launch();
        } else {
          // the second-pass increment is also kept apart (red) to subtract only it
          k_reduce_partials<<<Bi, 32, 0, c.st>>>(f->red, 33, 0, c.partial, col + 1, d_ids, 0);
          note_launch();
          k_combine<<<g, kVT, 0, c.st>>>(c.Rv, c.vs, f->V, vstr, f->red, 33, 0, nullptr, col + 1, -1.0, d_ids, N);
          note_launch();
        }
      }
      rc = sqnorm(c, c.Rv, c.vs, d_ids, Bi, S_NORM);
      if (rc) return rc;
      k_normalize<<<g, kVT, 0, c.st>>>(V_of(col + 1), c.Rv, vstr, c.vs, f->Hd, hld, col, f->scal, d_ids, N);
      note_launch();
      k_givens<<<(Bi + 63) / 64, 64, 0, c.st>>>(f->Hd, hld, f->cs, f->sn, f->gv, col, f->scal, d_ids, Bi);
      note_launch();
      ORBIT_CUDA_TRY(cudaGetLastError());
      rc = fetch_scal(c);
      if (rc) return rc;
      std::vector<int> keep;
      for (int o : inner) {
        iters[o]++;
        ncol_h[o] = col + 1;
        const double pres = f->h_scal[o * kScal + S_PRES];
        const bool brk = f->h_scal[o * kScal + S_BREAK] != 0.0;
        pres_h[o] = pres;
        if (!(pres <= atol[o] || brk)) keep.push_back(o);
        else est_done[o] = 1;
      }
      inner.swap(keep);
    }
    // x += V y for all orbits of this cycle
    B = (int)act.size();
    rc = upload_ids(c, act, d_ids);
    if (rc) return rc;
    ORBIT_CUDA_TRY(cudaMemcpyAsync(d_ncol, ncol_h.data(), sizeof(int) * f->n_orbits, cudaMemcpyHostToDevice, c.st));
    k_ysolve<<<(B + 63) / 64, 64, 0, c.st>>>(f->Hd, hld, f->gv, f->red, d_ncol, d_ids, B);
    note_launch();
    k_combine<<<vgrid(N, B), kVT, 0, c.st>>>(x, c.vs, f->V, vstr, f->red, 33, 0, d_ncol, 0, 1.0, d_ids, N);
    note_launch();
    if (trust_estimate) {
      // inner correction solves: accept the Arnoldi residual estimate
      std::vector<int> rest;
      for (int o : act) {
        if (est_done[o]) {
          conv[o] = 1;
          rn_out[o] = pres_h[o];
        } else {
          rest.push_back(o);
        }
      }
      act.swap(rest);
      if (act.empty()) break;
      B = (int)act.size();
      rc = upload_ids(c, act, d_ids);
      if (rc) return rc;
    }
    // true residual r = b - A x -> V0 (unnormalised) and its norm
    rc = matvec(c, x, c.vs, c.Rv, c.vs, d_ids, B, accurate_mv);
    if (rc) return rc;
    for (int o : act) matvecs[o]++;
    k_lincomb<<<vgrid(N, B), kVT, 0, c.st>>>(V_of(0), vstr, one, b, c.vs, mone, c.Rv, c.vs, d_ids, N);
    note_launch();
    rc = sqnorm(c, V_of(0), vstr, d_ids, B, S_NORM);
    if (rc) return rc;
    rc = fetch_scal(c);
    if (rc) return rc;
    std::vector<int> keep;
    for (int o : act) {
      const double rn = std::sqrt(std::max(f->h_scal[o * kScal + S_NORM], 0.0));
      rn_out[o] = rn;
      if (rn <= atol[o]) conv[o] = 1;
      else keep.push_back(o);
    }
    act.swap(keep);
  }
  return ORBIT_OK;
}

}  // namespace

// Periodic-orbit solve for the first n orbits.  e: caller (n, 8, N) cell order.
int orbit_solve_impl(orbit_factor_s* f, int n, const double* e_or_R, double dtau, const double* warm,
                     double tol, int maxiter, int restart, double* out, double* info, int trans,
                     cudaStream_t st) {
  orbit_symbolic_s* sy = f->sym;
  const int64_t N = sy->S.N;
  if (restart > f->restart_cap) restart = f->restart_cap;
  if (restart < 1) restart = 1;
  Ctx c;
  c.f = f; c.st = st; c.N = N; c.R = restart; c.hld = 33; c.mixed = f->precision == ORBIT_PREC_FP32;
  c.trans = trans;
  c.vs = 6 * N;
  c.Sv = f->tmpv; c.Xv = f->tmpv + N; c.Rv = f->tmpv + 2 * N; c.Dv = f->tmpv + 3 * N; c.Tv = f->tmpv + 4 * N;
  c.XS = f->tmpv + 6 * N * (int64_t)f->n_orbits;  // second region: 9N per orbit
  c.partial = f->red + 33 * (int64_t)f->n_orbits;
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->status, 0, sizeof(int), st));
  std::vector<int> all(n);
  for (int i = 0; i < n; ++i) all[i] = i;
  int* d_ids = f->orbit_ids;
  int rc = upload_ids(c, all, d_ids);
  if (rc) return rc;
  const dim3 g = vgrid(N, n);
  // forcing in permuted order
  k_perm_gather<<<g, kVT, 0, st>>>(f->E, 8 * N, e_or_R, 8 * N, 8, sy->d.perm, d_ids, N);
  note_launch();
  // s: forward x0 = 0, P_tau(x + dtau e); adjoint x8 = 0, P^T x + R
  Scal one{nullptr, 0, 0, 1.0}, zero{nullptr, 0, 0, 0.0};
  const int in = trans ? 8 : 0, outb = trans ? 0 : 8;
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->X, 0, sizeof(double) * 9 * N * n, st));
  const double fscale = trans ? 1.0 : dtau;
  std::vector<int> mv(f->n_orbits, 0), iters(f->n_orbits, 0), conv(f->n_orbits, 0), outer(f->n_orbits, 0);
  std::vector<double> rn(f->n_orbits, 0.0);
  // s = sweep of the forcing from zero.  In the mixed solves s only sets the
  // stopping tolerance (atol = tol ||s||; the block-cyclic refinement starts
  // from the forcing itself), so one FP32 sweep is enough there: its norm is
  // exact to ~1e-7 relative.  The FP64 solves sweep exactly.
  if (c.mixed) rc = launch_chain(f, n, d_ids, trans, 0, 8, f->E, fscale, st);
  else rc = chain_accurate(c, d_ids, n, f->E, fscale);
  if (rc) return rc;
  for (int o = 0; o < n; ++o) mv[o]++;
  k_lincomb<<<g, kVT, 0, st>>>(c.Sv, c.vs, one, f->X + outb * N, 9 * N, zero, nullptr, 0, d_ids, N);
  note_launch();
  rc = sqnorm(c, c.Sv, c.vs, d_ids, n, S_SN);
  if (rc) return rc;
  rc = fetch_scal(c);
  if (rc) return rc;
  std::vector<double> sn(n), atol(f->n_orbits, 0.0);
  std::vector<int> act, zero_orb;
  for (int o = 0; o < n; ++o) {
    sn[o] = std::sqrt(std::max(f->h_scal[o * kScal + S_SN], 0.0));
    if (!(sn[o] == sn[o]) || std::isinf(sn[o])) {
      set_last_error("non-finite forcing or solve result");
      return ORBIT_ERR_NOTFINITE;
    }
    if (sn[o] < 1e-30) zero_orb.push_back(o);
    else act.push_back(o);
    atol[o] = tol * sn[o];
  }
  // x0 = warm or s
  if (warm) {
    k_perm_gather<<<g, kVT, 0, st>>>(c.Xv, c.vs, warm, N, 1, sy->d.perm, d_ids, N);
    note_launch();
  } else {
    k_lincomb<<<g, kVT, 0, st>>>(c.Xv, c.vs, one, c.Sv, c.vs, zero, nullptr, 0, d_ids, N);
    note_launch();
  }
  bool mixed_done = false;
  if (!c.mixed) {
    rc = gmres(c, act, c.Sv, c.Xv, atol, maxiter, false, iters, conv, rn, mv, false);
    if (rc) return rc;
  } else if (!trans) {
    // Block-cyclic FP64 refinement.  The orbit is the solution of the eight
    // coupled bin equations A_tau c_{tau+1} = c_tau + dtau e_tau (c_0 := c_8);
    // their FP64 residual needs only stencil products.  Each correction solves
    // the same periodic problem with the residual as forcing, in FP32 (s_R by one
    // chained sweep, GMRES on (I - M~), recovery sweep), and the FP64 orbit
    // accumulates the corrections.  ||s_R|| is the reference's orbit residual
    // ||(I - M) c_0 - s|| of the current orbit (orbit.py:196-199).
    double* Cb = c.XS;                       // per orbit 9 vectors: c_1..c_8 in slots 1..8
    double* Rb = f->tmpv + 15 * N * (int64_t)f->n_orbits;  // per orbit 8 vectors
    ORBIT_CUDA_TRY(cudaMemsetAsync(Cb, 0, sizeof(double) * 9 * N * f->n_orbits, st));
    std::vector<int> oact = act;
    if (warm && !oact.empty()) {
      // start from the FP32 sweep of the warm start
      const int B = (int)oact.size();
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      k_lincomb<<<vgrid(N, B), kVT, 0, st>>>(f->X, 9 * N, one, c.Xv, c.vs, zero, nullptr, 0, d_ids, N);
      note_launch();
      rc = launch_chain(f, B, d_ids, 0, 0, 8, f->E, dtau, st);
      if (rc) return rc;
      for (int t = 1; t <= 8; ++t) {
        k_lincomb<<<vgrid(N, B), kVT, 0, st>>>(Cb + t * N, 9 * N, one, f->X + t * N, 9 * N, zero, nullptr, 0,
                                               d_ids, N);
        note_launch();
      }
      for (int o : oact) mv[o]++;
    }
    const int max_outer = 8;
    for (int it = 0; it <= max_outer && !oact.empty(); ++it) {
      const int B = (int)oact.size();
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      const dim3 gb = vgrid(N, B);
      k_block_resid<<<gb, kVT, 0, st>>>(Rb, f->E, dtau, Cb, f->A_stencil, sy->d.perm, sy->d.iperm, sy->S.nz,
                                        sy->S.ny, sy->S.nx, sy->S.periodic_x, d_ids, f->set_of);
      note_launch();
      if (it == 0 && !warm) {
        // from c = 0 the residual forcing is dtau e itself, whose sweep is the
        // s computed above: reuse it
        k_lincomb<<<gb, kVT, 0, st>>>(c.Dv, c.vs, one, c.Sv, c.vs, zero, nullptr, 0, d_ids, N);
        note_launch();
      } else {
        ORBIT_CUDA_TRY(cudaMemsetAsync(f->X, 0, sizeof(double) * 9 * N * f->n_orbits, st));
        rc = launch_chain(f, B, d_ids, 0, 0, 8, Rb, 1.0, st);
        if (rc) return rc;
        for (int o : oact) mv[o]++;
        k_lincomb<<<gb, kVT, 0, st>>>(c.Dv, c.vs, one, f->X + 8 * N, 9 * N, zero, nullptr, 0, d_ids, N);
        note_launch();
      }
      rc = sqnorm(c, c.Dv, c.vs, d_ids, B, S_TMP);
      if (rc) return rc;
      rc = fetch_scal(c);
      if (rc) return rc;
      std::vector<int> keep;
      std::vector<double> itol(f->n_orbits, 0.0);
      for (int o : oact) {
        const double r = std::sqrt(std::max(f->h_scal[o * kScal + S_TMP], 0.0));
        rn[o] = r;
        if (r <= atol[o]) {
          conv[o] = 1;
        } else if (it < max_outer) {
          keep.push_back(o);
          itol[o] = std::max(atol[o] * 0.5, 1e-4 * r);
        }
      }
      oact.swap(keep);
      if (oact.empty()) break;
      const int B2 = (int)oact.size();
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      double* xcorr = f->tmpv + 5 * N;
      k_lincomb<<<vgrid(N, B2), kVT, 0, st>>>(xcorr, c.vs, zero, nullptr, 0, zero, nullptr, 0, d_ids, N);
      note_launch();
      std::vector<int> cin(f->n_orbits, 0);
      std::vector<double> rin(f->n_orbits, 0.0);
      rc = gmres(c, oact, c.Dv, xcorr, itol, maxiter, false, iters, cin, rin, mv, true, true);
      if (rc) return rc;
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      // corrections of every bin: recovery sweep from delta_0 with the residual forcing
      ORBIT_CUDA_TRY(cudaMemsetAsync(f->X, 0, sizeof(double) * 9 * N * f->n_orbits, st));
      k_lincomb<<<vgrid(N, B2), kVT, 0, st>>>(f->X, 9 * N, one, xcorr, c.vs, zero, nullptr, 0, d_ids, N);
      note_launch();
      rc = launch_chain(f, B2, d_ids, 0, 0, 8, Rb, 1.0, st);
      if (rc) return rc;
      for (int o : oact) mv[o]++;
      for (int t = 1; t <= 8; ++t) {
        k_lincomb<<<vgrid(N, B2), kVT, 0, st>>>(Cb + t * N, 9 * N, one, Cb + t * N, 9 * N, one, f->X + t * N,
                                                9 * N, d_ids, N);
        note_launch();
      }
      for (int o : oact) outer[o]++;
    }
    // orbit [c_8, c_1, ..., c_8] into the chain buffer
    rc = upload_ids(c, all, d_ids);
    if (rc) return rc;
    for (int t = 0; t <= 8; ++t) {
      k_lincomb<<<g, kVT, 0, st>>>(f->X + t * N, 9 * N, one, Cb + (t == 0 ? 8 : t) * N, 9 * N, zero, nullptr,
                                   0, d_ids, N);
      note_launch();
    }
    // periodicity of the exact sweep from c_0: ||c_8' - c_0|| = ||(I - M) c_0 - s||
    k_lincomb<<<g, kVT, 0, st>>>(c.Tv, c.vs, one, c.Dv, c.vs, zero, nullptr, 0, d_ids, N);
    note_launch();
    mixed_done = true;
  } else {
    // Block-cyclic FP64 refinement of the transposed problem, the mirror of the
    // forward one: the adjoint orbit solves the eight coupled equations
    // A_tau^T (lam_tau - R_tau) = lam_{tau+1} (lam_8 := lam_0), whose FP64
    // residual rho needs only stencil products (k_block_resid_T).  A correction
    // delta solves the same periodic problem with rho as forcing,
    // delta_tau = P_tau^T (delta_{tau+1} + rho_tau), in FP32: s_rho by one
    // transposed sweep, GMRES on (I - M~^T), one recovery sweep; the FP64 orbit
    // accumulates the corrections.  ||s_rho|| is the adjoint residual
    // ||(I - M^T) lam_0 - s|| of the current orbit.
    double* Lb = c.XS;                                     // per orbit 9: lam_0..lam_7 in slots 0..7
    double* Rs = f->tmpv + 15 * N * (int64_t)f->n_orbits;  // per orbit 8: shifted residual forcing
    double* rho7 = c.Xv;                                   // per orbit: rho_7 (stride vs)
    ORBIT_CUDA_TRY(cudaMemsetAsync(Lb, 0, sizeof(double) * 9 * N * f->n_orbits, st));
    std::vector<int> oact = act;
    if (warm && !oact.empty()) {
      // start from the FP32 transposed sweep of the warm start:
      // lam_tau = X[tau] + R_tau (tau = 1..7), lam_0 = X[0]
      const int B = (int)oact.size();
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      ORBIT_CUDA_TRY(cudaMemsetAsync(f->X, 0, sizeof(double) * 9 * N * f->n_orbits, st));
      k_lincomb<<<vgrid(N, B), kVT, 0, st>>>(f->X + 8 * N, 9 * N, one, c.Xv, c.vs, zero, nullptr, 0, d_ids, N);
      note_launch();
      rc = launch_chain(f, B, d_ids, 1, 0, 8, f->E, 1.0, st);
      if (rc) return rc;
      for (int t = 0; t < 8; ++t) {
        k_lincomb<<<vgrid(N, B), kVT, 0, st>>>(Lb + t * N, 9 * N, one, f->X + t * N, 9 * N, t == 0 ? zero : one,
                                               t == 0 ? nullptr : f->E + t * N, 8 * N, d_ids, N);
        note_launch();
      }
      for (int o : oact) mv[o]++;
    }
    const int max_outer = 8;
    for (int it = 0; it <= max_outer && !oact.empty(); ++it) {
      const int B = (int)oact.size();
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      const dim3 gb = vgrid(N, B);
      k_block_resid_T<<<gb, kVT, 0, st>>>(Rs, rho7, c.vs, f->E, Lb, f->A_stencil, sy->d.perm, sy->d.iperm, sy->S.nz,
                                          sy->S.ny, sy->S.nx, sy->S.periodic_x, d_ids, f->set_of);
      note_launch();
      if (it == 0 && !warm) {
        // from lam = 0 the residual is rho_tau = A_tau^T R_tau, and the sweep
        // of it ends (slot 0) where the sweep of the receptors s ends: reuse s
        k_lincomb<<<gb, kVT, 0, st>>>(c.Dv, c.vs, one, c.Sv, c.vs, zero, nullptr, 0, d_ids, N);
        note_launch();
      } else {
        // s_rho: transposed sweep from X[8] = rho_7 with the shifted forcing
        ORBIT_CUDA_TRY(cudaMemsetAsync(f->X, 0, sizeof(double) * 9 * N * f->n_orbits, st));
        k_lincomb<<<gb, kVT, 0, st>>>(f->X + 8 * N, 9 * N, one, rho7, c.vs, zero, nullptr, 0, d_ids, N);
        note_launch();
        rc = launch_chain(f, B, d_ids, 1, 0, 8, Rs, 1.0, st);
        if (rc) return rc;
        for (int o : oact) mv[o]++;
        k_lincomb<<<gb, kVT, 0, st>>>(c.Dv, c.vs, one, f->X, 9 * N, zero, nullptr, 0, d_ids, N);
        note_launch();
      }
      rc = sqnorm(c, c.Dv, c.vs, d_ids, B, S_TMP);
      if (rc) return rc;
      rc = fetch_scal(c);
      if (rc) return rc;
      std::vector<int> keep;
      std::vector<double> itol(f->n_orbits, 0.0);
      for (int o : oact) {
        const double r = std::sqrt(std::max(f->h_scal[o * kScal + S_TMP], 0.0));
        rn[o] = r;
        if (r <= atol[o]) {
          conv[o] = 1;
        } else if (it < max_outer) {
          keep.push_back(o);
          itol[o] = std::max(atol[o] * 0.5, 1e-4 * r);
        }
      }
      oact.swap(keep);
      if (oact.empty()) break;
      const int B2 = (int)oact.size();
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      double* xcorr = f->tmpv + 5 * N;
      k_lincomb<<<vgrid(N, B2), kVT, 0, st>>>(xcorr, c.vs, zero, nullptr, 0, zero, nullptr, 0, d_ids, N);
      note_launch();
      std::vector<int> cin(f->n_orbits, 0);
      std::vector<double> rin(f->n_orbits, 0.0);
      rc = gmres(c, oact, c.Dv, xcorr, itol, maxiter, false, iters, cin, rin, mv, true, true);
      if (rc) return rc;
      rc = upload_ids(c, oact, d_ids);
      if (rc) return rc;
      // corrections of every bin: recovery sweep from X[8] = delta_0 + rho_7
      ORBIT_CUDA_TRY(cudaMemsetAsync(f->X, 0, sizeof(double) * 9 * N * f->n_orbits, st));
      k_lincomb<<<vgrid(N, B2), kVT, 0, st>>>(f->X + 8 * N, 9 * N, one, xcorr, c.vs, one, rho7, c.vs, d_ids, N);
      note_launch();
      rc = launch_chain(f, B2, d_ids, 1, 0, 8, Rs, 1.0, st);
      if (rc) return rc;
      for (int o : oact) mv[o]++;
      for (int t = 0; t < 8; ++t) {
        k_lincomb<<<vgrid(N, B2), kVT, 0, st>>>(Lb + t * N, 9 * N, one, Lb + t * N, 9 * N, one, f->X + t * N,
                                                9 * N, d_ids, N);
        note_launch();
      }
      for (int o : oact) outer[o]++;
    }
    // adjoint orbit [lam_0, ..., lam_7, lam_0] into the chain buffer
    rc = upload_ids(c, all, d_ids);
    if (rc) return rc;
    for (int t = 0; t <= 8; ++t) {
      k_lincomb<<<g, kVT, 0, st>>>(f->X + t * N, 9 * N, one, Lb + (t == 8 ? 0 : t) * N, 9 * N, zero, nullptr, 0,
                                   d_ids, N);
      note_launch();
    }
    // periodicity from the last residual sweep, as in the forward solve
    k_lincomb<<<g, kVT, 0, st>>>(c.Tv, c.vs, one, c.Dv, c.vs, zero, nullptr, 0, d_ids, N);
    note_launch();
    mixed_done = true;
  }
  // recovery: chain with forcing from x
  rc = upload_ids(c, all, d_ids);
  if (rc) return rc;
  if (!mixed_done) {
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->X, 0, sizeof(double) * 9 * N * n, st));
  k_lincomb<<<g, kVT, 0, st>>>(f->X + in * N, 9 * N, one, c.Xv, c.vs, zero, nullptr, 0, d_ids, N);
  note_launch();
  if (!trans) {
    rc = chain_accurate(c, d_ids, n, f->E, fscale);
    if (rc) return rc;
  } else {
    // adjoint unroll: lam_tau = P_tau^T lam_{tau+1} + R_tau for tau = 7..1, lam_8 = lam_0
    rc = chain_accurate(c, d_ids, n, f->E, fscale, 1, 8);
    if (rc) return rc;
    // X[tau] for tau = 2..7 hold P^T(...) without R: add R_tau (X[1] already has it)
    for (int t = 2; t < 8; ++t) {
      k_lincomb<<<g, kVT, 0, st>>>(f->X + t * N, 9 * N, one, f->X + t * N, 9 * N, one, f->E + t * N, 8 * N, d_ids, N);
      note_launch();
    }
  }
  for (int o = 0; o < n; ++o) mv[o]++;
  // periodicity: forward ||X8 - X0|| / (||X0|| + 1e-30); adjoint: ||P0^T lam1 + R0 - lam0|| / ...
  if (!trans) {
    Scal mone{nullptr, 0, 0, -1.0};
    k_lincomb<<<g, kVT, 0, st>>>(c.Tv, c.vs, one, f->X + 8 * N, 9 * N, mone, f->X, 9 * N, d_ids, N);
    note_launch();
  } else {
    // lam0_check = P_0^T lam_1 + R_0 computed in place into X[0], then X[0] = lam_0
    Scal mone{nullptr, 0, 0, -1.0};
    rc = chain_accurate(c, d_ids, n, f->E, fscale, 0, 1);
    if (rc) return rc;
    k_lincomb<<<g, kVT, 0, st>>>(c.Tv, c.vs, one, f->X, 9 * N, mone, c.Xv, c.vs, d_ids, N);
    note_launch();
    k_lincomb<<<g, kVT, 0, st>>>(f->X, 9 * N, one, c.Xv, c.vs, zero, nullptr, 0, d_ids, N);
    note_launch();
    k_lincomb<<<g, kVT, 0, st>>>(f->X + 8 * N, 9 * N, one, c.Xv, c.vs, zero, nullptr, 0, d_ids, N);
    note_launch();
  }
  }
  rc = sqnorm(c, c.Tv, c.vs, d_ids, n, S_TMP);
  if (rc) return rc;
  rc = sqnorm(c, f->X, 9 * N, d_ids, n, S_H0);
  if (rc) return rc;
  k_count_neg<<<dim3(kRedBlocks, n), kVT, 0, st>>>(c.partial, f->X, 9 * N, 9 * N, d_ids);
  note_launch();
  k_reduce_partials<<<n, 32, 0, st>>>(f->scal, kScal, S_NEG, c.partial, 1, d_ids, 0);
  note_launch();
  // outputs in cell order
  k_perm_scatter<<<g, kVT, 0, st>>>(out, 9 * N, f->X, 9 * N, 9, sy->d.perm, d_ids, N);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  rc = fetch_scal(c);
  if (rc) return rc;
  for (int o = 0; o < n; ++o) {
    double* inf = info + o * 8;
    const bool z = sn[o] < 1e-30;
    const double per = std::sqrt(std::max(f->h_scal[o * kScal + S_TMP], 0.0)) /
                       (std::sqrt(std::max(f->h_scal[o * kScal + S_H0], 0.0)) + 1e-30);
    inf[0] = iters[o];
    inf[1] = z ? 0.0 : rn[o] / sn[o];
    inf[2] = z ? 0.0 : per;
    inf[3] = z ? 0.0 : f->h_scal[o * kScal + S_NEG] / (9.0 * N);
    inf[4] = z ? 1.0 : (double)conv[o];
    inf[5] = sn[o];
    inf[6] = outer[o];
    inf[7] = mv[o];
  }
  if (!zero_orb.empty()) {
    // zero forcing -> zero orbit (orbit.py:155-160)
    for (int o : zero_orb)
      ORBIT_CUDA_TRY(cudaMemsetAsync(out + (int64_t)o * 9 * N, 0, sizeof(double) * 9 * N, st));
  }
  for (int o : act)
    if (!conv[o]) {
      set_last_error("GMRES did not converge for at least one orbit");
      return ORBIT_ERR_NOCONV;
    }
  return ORBIT_OK;
}

}  // namespace orbit

namespace orbit {

// Chain application through the C ABI: x_out = P_{tau1-1}..P_{tau0} x_in (or the transposed chain),
// with optional forcing and, for FP32 factors, optional FP64 refinement of every bin solve.
int chain_apply_impl(orbit_factor_s* f, int n, int trans, int tau0, int tau1, const double* x_in,
                     double* x_out, const double* forcing, double fscale, int refine, cudaStream_t st) {
  orbit_symbolic_s* sy = f->sym;
  const int64_t N = sy->S.N;
  Ctx c;
  c.f = f; c.st = st; c.N = N; c.R = 1; c.hld = 33;
  c.mixed = f->precision == ORBIT_PREC_FP32 && refine;
  c.trans = trans;
  c.vs = 6 * N;
  c.Sv = f->tmpv; c.Xv = f->tmpv + N; c.Rv = f->tmpv + 2 * N; c.Dv = f->tmpv + 3 * N; c.Tv = f->tmpv + 4 * N;
  c.XS = f->tmpv + 6 * N * (int64_t)f->n_orbits;
  c.partial = f->red + 33 * (int64_t)f->n_orbits;
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->status, 0, sizeof(int), st));
  std::vector<int> all(n);
  for (int i = 0; i < n; ++i) all[i] = i;
  int* d_ids = f->orbit_ids;
  int rc = upload_ids(c, all, d_ids);
  if (rc) return rc;
  const dim3 g = vgrid(N, n);
  const int in = trans ? tau1 : tau0, out = trans ? tau0 : tau1;
  k_perm_gather<<<g, kVT, 0, st>>>(f->X + (int64_t)in * N, 9 * N, x_in, N, 1, sy->d.perm, d_ids, N);
  note_launch();
  const double* E = nullptr;
  if (forcing) {
    k_perm_gather<<<g, kVT, 0, st>>>(f->E, 8 * N, forcing, 8 * N, 8, sy->d.perm, d_ids, N);
    note_launch();
    E = f->E;
  }
  ORBIT_CUDA_TRY(cudaGetLastError());
  rc = chain_accurate(c, d_ids, n, E, fscale, tau0, tau1);
  if (rc) return rc;
  k_perm_scatter<<<g, kVT, 0, st>>>(x_out, N, f->X + (int64_t)out * N, 9 * N, 1, sy->d.perm, d_ids, N);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return fetch_scal(c);
}

}  // namespace orbit
