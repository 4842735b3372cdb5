// K4: chained supernodal triangular solves through all diurnal bins in one
// persistent launch.
//
// Replaces the reference's eight sequential lu.solve calls per monodromy
// application (apply_monodromy, orbit/core/orbit.py:99-107; compute_s,
// orbit.py:110-120; the recovery sweep orbit.py:188-193) and their
// transposed twins (orbit/core/orbit_adjoint.py:36-67, 127-134).
//
// Work is a static list of tasks (bin, supernode, row chunk, orbit), ordered
// bin by bin: the forward sweep from the leaves to the root, then the
// backward sweep from the root to the leaves.  CTAs claim tasks in that order
// from an atomic counter and wait (bounded spin, acquire loads) only on the
// per-supernode completion counters of the tasks a task reads from: its
// children's update vectors, the previous bin's solution on its own rows, or
// its parent's backward result.  Since every dependency precedes its
// dependant in claim order and the grid is sized to be co-resident, the
// earliest unfinished task can always run.  A wait that exceeds its
// iteration limit sets ORBIT_ERR_TIMEOUT in the status word and every CTA
// leaves the loop.
#include <cuda_runtime.h>

#include "common.cuh"
#include "handles.h"

namespace orbit {

namespace {

constexpr int kSolveThreads = 256;
constexpr int kWarps = kSolveThreads / 32;

template <typename T>
struct ChainDev {
  const int32_t *first, *n, *m, *parent, *child, *uidx, *rel, *ldn, *ldm;
  const int32_t *nch_f, *nch_b;
  const int64_t *uoff, *fac_off, *woff;
  const int4* items;
  const int32_t* phase_off;
  int nphase, items_per_bin, nsuper;
  int64_t N, fac_size, w_size;
  const T* factors;
  double* X;
  const double* E;
  double escale;
  double* Y;
  double* W;
  int* counters;
  int* task_counter;
  int* status;
  const int* orbit_ids;
  int B, tau0, tau1, trans;
  int total;
  long long spin_limit;
};

__device__ __forceinline__ bool wait_ge(const int* p, int target, int* status, long long limit) {
  long long it = 0;
  while (ld_acquire(p) < target) {
    if (ld_volatile(status) != 0) return false;
    if (++it > limit) {
      raise_status(status, ORBIT_ERR_TIMEOUT);
      return false;
    }
    __nanosleep(100);
  }
  return true;
}

template <typename T>
__device__ __forceinline__ T dot_row(const T* __restrict__ a, const T* v, int len, int lane) {
  T acc0 = T(0), acc1 = T(0), acc2 = T(0), acc3 = T(0);
  int j = lane;
  for (; j + 96 < len; j += 128) {
    T a0 = __ldg(a + j), a1 = __ldg(a + j + 32), a2 = __ldg(a + j + 64), a3 = __ldg(a + j + 96);
    acc0 = fma(a0, v[j], acc0);
    acc1 = fma(a1, v[j + 32], acc1);
    acc2 = fma(a2, v[j + 64], acc2);
    acc3 = fma(a3, v[j + 96], acc3);
  }
  for (; j < len; j += 32) acc0 = fma(__ldg(a + j), v[j], acc0);
  return warp_sum((acc0 + acc1) + (acc2 + acc3));
}

// Forward step of one supernode (L, or U^T when trans) for output rows
// [r0, r1): gathers its right-hand side (own entries of Xin, plus forcing) and
// the children's update vectors into `vec`, then one dense GEMV.  Ends with a
// block barrier.
template <typename T>
__device__ void fwd_node(const ChainDev<T>& D, int o, int tau, int s, int r0, int r1, bool trans,
                         T* vec, T* red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t N = D.N;
  const int n = D.n[s], m = D.m[s], first = D.first[s];
  const int ldn = D.ldn[s], ldm = D.ldm[s];
  const T* SQ = D.factors + (int64_t)(o * 8 + tau) * D.fac_size + D.fac_off[s];
  double* Yo = D.Y + (int64_t)o * N;
  double* Wo = D.W + (int64_t)o * D.w_size;
  const int bin_in = trans ? tau + 1 : tau;
  const double* Xin = D.X + ((int64_t)o * 9 + bin_in) * N;
  const double* Ein = nullptr;
  if (D.E) {
    if (!trans) Ein = D.E + ((int64_t)o * 8 + tau) * N;
    else if (tau + 1 < D.tau1) Ein = D.E + ((int64_t)o * 8 + tau + 1) * N;
  }
  for (int i = tid; i < n + m; i += kSolveThreads) {
    double v = 0.0;
    if (i < n) {
      v = Xin[first + i];
      if (Ein) v += D.escale * Ein[first + i];
    }
    vec[i] = (T)v;
  }
  for (int q2 = 0; q2 < 2; ++q2) {
    __syncthreads();
    const int c = D.child[2 * s + q2];
    if (c < 0) continue;
    const int mc = D.m[c];
    const int32_t* rel = D.rel + D.uoff[c];
    const double* wc = Wo + D.woff[c];
    for (int j = tid; j < mc; j += kSolveThreads) vec[rel[j]] += (T)wc[j];
  }
  __syncthreads();
  if (!trans) {
    // rows of [SQ; Pb]: row i < n uses the strict lower part (unit diagonal)
    for (int i = r0 + warp; i < r1; i += kWarps) {
      const int len = i < n ? i : n;
      T acc = dot_row(SQ + (int64_t)i * ldn, vec, len, lane);
      if (lane == 0) {
        if (i < n) Yo[first + i] = (double)(vec[i] + acc);
        else Wo[D.woff[s] + (i - n)] = (double)(vec[i] + acc);
      }
    }
  } else {
    // columns of [upper(SQ) | Qr]
    const T* Qr = SQ + (int64_t)(n + m) * ldn;
    for (int cb = r0; cb < r1; cb += 32) {
      const int c = cb + lane;
      T acc = T(0);
      if (c < r1) {
        if (c < n) {
          for (int i = warp; i <= c; i += kWarps) acc = fma(__ldg(SQ + (int64_t)i * ldn + c), vec[i], acc);
        } else {
          const int u = c - n;
          for (int i = warp; i < n; i += kWarps) acc = fma(__ldg(Qr + (int64_t)i * ldm + u), vec[i], acc);
        }
      }
      red[warp * 32 + lane] = acc;
      __syncthreads();
      if (warp == 0 && c < r1) {
        T sum = T(0);
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sum += red[w * 32 + lane];
        if (c < n) Yo[first + c] = (double)sum;
        else Wo[D.woff[s] + (c - n)] = (double)(vec[c] + sum);
      }
      __syncthreads();
    }
  }
  __syncthreads();
}

// Backward step of one supernode (U, or L^T when trans) for rows [r0, r1):
// own forward result plus the ancestors' solution.  Ends with a block barrier.
template <typename T>
__device__ void bwd_node(const ChainDev<T>& D, int o, int tau, int s, int r0, int r1, bool trans,
                         T* vec, T* red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t N = D.N;
  const int n = D.n[s], m = D.m[s], first = D.first[s];
  const int ldn = D.ldn[s], ldm = D.ldm[s];
  const T* SQ = D.factors + (int64_t)(o * 8 + tau) * D.fac_size + D.fac_off[s];
  const double* Yo = D.Y + (int64_t)o * N;
  const int bin_out = trans ? tau : tau + 1;
  double* Xout = D.X + ((int64_t)o * 9 + bin_out) * N;
  const int32_t* ui = D.uidx + D.uoff[s];
  for (int i = tid; i < n + m; i += kSolveThreads) vec[i] = (T)(i < n ? Yo[first + i] : Xout[ui[i - n]]);
  __syncthreads();
  if (!trans) {
    const T* Qr = SQ + (int64_t)(n + m) * ldn;
    for (int i = r0 + warp; i < r1; i += kWarps) {
      const T* row = SQ + (int64_t)i * ldn;
      T acc0 = T(0), acc1 = T(0);
      for (int j = i + lane; j < n; j += 32) acc0 = fma(__ldg(row + j), vec[j], acc0);
      const T* qrow = Qr + (int64_t)i * ldm;
      int j = lane;
      for (; j + 32 < m; j += 64) {
        acc1 = fma(__ldg(qrow + j), vec[n + j], acc1);
        acc0 = fma(__ldg(qrow + j + 32), vec[n + j + 32], acc0);
      }
      for (; j < m; j += 32) acc1 = fma(__ldg(qrow + j), vec[n + j], acc1);
      T acc = warp_sum(acc0 + acc1);
      if (lane == 0) Xout[first + i] = (double)acc;
    }
  } else {
    // columns of [SQ_strict_lower ; Pb] with unit diagonal
    for (int cb = r0; cb < r1; cb += 32) {
      const int c = cb + lane;
      T acc = T(0);
      if (c < r1) {
        for (int i = c + 1 + warp; i < n + m; i += kWarps) acc = fma(__ldg(SQ + (int64_t)i * ldn + c), vec[i], acc);
      }
      red[warp * 32 + lane] = acc;
      __syncthreads();
      if (warp == 0 && c < r1) {
        T sum = vec[c];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sum += red[w * 32 + lane];
        Xout[first + c] = (double)sum;
      }
      __syncthreads();
    }
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kSolveThreads) k_chain(ChainDev<T> D) {
  extern __shared__ unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);      // kWarps * 32
  T* vec = red + kWarps * 32;                    // front-sized vector
  __shared__ int s_task;
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  const int per_bin = D.items_per_bin * D.B;
  for (;;) {
    if (tid == 0) {
      s_task = atomicAdd(D.task_counter, 1);
      s_ok = ld_volatile(D.status) == 0;
    }
    __syncthreads();
    const int t = s_task;
    if (t >= D.total || !s_ok) break;
    const int q = t / per_bin;
    const int r = t - q * per_bin;
    const int tau = D.trans ? (D.tau1 - 1 - q) : (D.tau0 + q);
    int p = 0;
    while (D.phase_off[p + 1] * D.B <= r) ++p;
    const int rr = r - D.phase_off[p] * D.B;
    const int cnt = D.phase_off[p + 1] - D.phase_off[p];
    const int oi = rr / cnt;
    const int4 it = D.items[D.phase_off[p] + (rr - oi * cnt)];
    const int o = D.orbit_ids[oi];
    const int s = it.x, kind = it.w;
    const bool fwd = (kind & 1) == 0;        // kinds 0, 2, 4, 6
    const bool trans = kind == 2 || kind == 3 || kind == 6 || kind == 7;
    const bool subtree = kind >= 4;
    int* cbase = D.counters + (int64_t)o * 8 * 2 * D.nsuper;
    // ---- dependencies ----
    if (tid == 0) {
      bool ok = true;
      if (fwd) {
        if (!subtree)
          for (int q2 = 0; q2 < 2 && ok; ++q2) {
            const int c = D.child[2 * s + q2];
            if (c >= 0) ok = wait_ge(cbase + (tau * 2 + 0) * D.nsuper + c, D.nch_f[c], D.status, D.spin_limit);
          }
        if (ok && !trans && tau > D.tau0)
          ok = wait_ge(cbase + ((tau - 1) * 2 + 1) * D.nsuper + s, D.nch_b[s], D.status, D.spin_limit);
        if (ok && trans && tau < D.tau1 - 1)
          ok = wait_ge(cbase + ((tau + 1) * 2 + 1) * D.nsuper + s, D.nch_b[s], D.status, D.spin_limit);
      } else {
        const int par = D.parent[s];
        if (par < 0)
          ok = wait_ge(cbase + (tau * 2 + 0) * D.nsuper + s, D.nch_f[s], D.status, D.spin_limit);
        else
          ok = wait_ge(cbase + (tau * 2 + 1) * D.nsuper + par, D.nch_b[par], D.status, D.spin_limit);
      }
      s_ok = ok;
      __threadfence();
    }
    __syncthreads();
    if (!s_ok) break;
    if (!subtree) {
      if (fwd) fwd_node(D, o, tau, s, it.y, it.z, trans, vec, red);
      else bwd_node(D, o, tau, s, it.y, it.z, trans, vec, red);
    } else if (fwd) {
      // postorder: every child before its parent
      for (int d = it.y; d <= s; ++d)
        fwd_node(D, o, tau, d, 0, trans ? D.n[d] + D.m[d] : D.n[d] + D.m[d], trans, vec, red);
    } else {
      // reverse postorder: every parent before its children
      for (int d = s; d >= it.y; --d) bwd_node(D, o, tau, d, 0, D.n[d], trans, vec, red);
    }
    if (tid == 0) {
      __threadfence();
      red_release_add(cbase + (tau * 2 + (fwd ? 0 : 1)) * D.nsuper + s, 1);
    }
  }
}

// x[tau0] += escale * E[tau0] (forcing of the transposed chain's last bin)
__global__ void k_add_forcing(double* X, const double* E, const int* orbit_ids, int64_t N, int tau0,
                              double escale) {
  const int o = orbit_ids[blockIdx.y];
  double* x = X + ((int64_t)o * 9 + tau0) * N;
  const double* e = E + ((int64_t)o * 8 + tau0) * N;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += escale * e[i];
}

template <typename T>
int launch_chain_t(orbit_factor_s* f, double* X, int B, const int* d_orbit_ids, int trans, int tau0,
                   int tau1, const double* E, double escale, cudaStream_t st) {
  orbit_symbolic_s* sy = f->sym;
  const Symbolic& S = sy->S;
  ChainDev<T> D;
  D.first = sy->d.first; D.n = sy->d.n; D.m = sy->d.m; D.parent = sy->d.parent;
  D.child = sy->d.child; D.uidx = sy->d.uidx; D.rel = sy->d.rel; D.ldn = sy->d.ldn; D.ldm = sy->d.ldm;
  D.nch_f = trans ? sy->d.nchunk_fwdT : sy->d.nchunk_fwd;
  D.nch_b = trans ? sy->d.nchunk_bwdT : sy->d.nchunk_bwd;
  D.uoff = sy->d.uoff; D.fac_off = sy->d.fac_off; D.woff = sy->d.woff;
  D.items = trans ? sy->d.sitems + S.items_per_bin : sy->d.sitems;
  D.phase_off = trans ? sy->d.phase_offT : sy->d.phase_off;
  D.nphase = 2 * S.nlevels;
  D.items_per_bin = trans ? S.items_per_binT : S.items_per_bin;
  D.nsuper = S.nsuper;
  D.N = S.N; D.fac_size = S.fac_size; D.w_size = S.w_size;
  D.factors = reinterpret_cast<const T*>(f->factors);
  D.X = X; D.E = E; D.escale = escale; D.Y = f->Ybuf; D.W = f->Wbuf;
  D.counters = f->counters; D.task_counter = f->task_counter; D.status = f->status;
  D.orbit_ids = d_orbit_ids; D.B = B; D.tau0 = tau0; D.tau1 = tau1; D.trans = trans;
  D.total = (tau1 - tau0) * D.items_per_bin * B;
  D.spin_limit = 4000000LL;  // bounded: a few seconds of 100 ns sleeps
  if (D.total <= 0) return ORBIT_OK;
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->counters, 0, sizeof(int) * (size_t)f->n_orbits * 16 * S.nsuper, st));
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->task_counter, 0, sizeof(int), st));
  const size_t smem = sizeof(T) * ((size_t)kWarps * 32 + S.max_front + 8);
  ORBIT_CUDA_TRY(cudaFuncSetAttribute(k_chain<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 0, occ = 0;
  ORBIT_CUDA_TRY(cudaGetDevice(&dev));
  ORBIT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  ORBIT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_chain<T>, kSolveThreads, smem));
  if (occ < 1) {
    set_last_error("chain kernel cannot be resident");
    return ORBIT_ERR_INTERNAL;
  }
  int grid = sms * occ;
  if (grid > D.total) grid = D.total;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (f->prof_on) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
  }
  k_chain<T><<<grid, kSolveThreads, smem, st>>>(D);
  note_launch();
  if (f->prof_on) {
    cudaEventRecord(e1, st);
    f->prof_chain.push_back({e0, e1});
    f->prof_chain_bytes += (double)B * (tau1 - tau0) * S.fac_nnz * sizeof(T);
  }
  ORBIT_CUDA_TRY(cudaGetLastError());
  if (trans && E) {
    dim3 g((unsigned)((S.N + 255) / 256), B);
    k_add_forcing<<<g, 256, 0, st>>>(X, E, d_orbit_ids, S.N, tau0, escale);
    note_launch();
    ORBIT_CUDA_TRY(cudaGetLastError());
  }
  return ORBIT_OK;
}

}  // namespace

// Run the chain on f->X (per orbit 9 vectors in permuted order).  Forward:
// reads X[tau0], writes X[tau0+1..tau1].  Transposed: reads X[tau1], writes
// X[tau1-1..tau0].  E (permuted, per orbit 8 vectors) may be null.
int launch_chain_x(orbit_factor_s* f, double* X, int B, const int* d_orbit_ids, int trans, int tau0,
                   int tau1, const double* E, double escale, cudaStream_t st) {
  if (f->precision == ORBIT_PREC_FP32)
    return launch_chain_t<float>(f, X, B, d_orbit_ids, trans, tau0, tau1, E, escale, st);
  return launch_chain_t<double>(f, X, B, d_orbit_ids, trans, tau0, tau1, E, escale, st);
}

int launch_chain(orbit_factor_s* f, int B, const int* d_orbit_ids, int trans, int tau0, int tau1,
                 const double* E, double escale, cudaStream_t st) {
  return launch_chain_x(f, f->X, B, d_orbit_ids, trans, tau0, tau1, E, escale, st);
}

}  // namespace orbit
