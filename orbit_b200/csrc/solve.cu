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
//
// Ordering: a task's results are written by all its threads, then a block
// barrier, then one thread's red.release.gpu on the completion counter; the
// consumer's thread polls with ld.acquire.gpu, then a block barrier, then all
// its threads read.  Release and acquire are cumulative over the barriers'
// CTA-scope ordering, so no separate fence is needed on either side.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "handles.h"

namespace orbit {

namespace {

#ifndef ORBIT_SOLVE_THREADS
#define ORBIT_SOLVE_THREADS 128
#endif
// CTAs per SM the chain kernels are compiled for, per precision: FP32 at 10
// (48 registers) hides more of the per-task latency than at 8 (64 registers),
// 4 % faster on a 12-orbit chain even with the few spills it costs; FP64 at 7
// (72 registers), which holds twelve 16-byte loads per lane in flight
#ifndef ORBIT_SOLVE_MINB
#define ORBIT_SOLVE_MINB 7
#endif
#ifndef ORBIT_SOLVE_MINB_FP32
#define ORBIT_SOLVE_MINB_FP32 10
#endif
constexpr int kSolveThreads = ORBIT_SOLVE_THREADS;
constexpr int kMaxPhases = 96;  // 2 x tree levels
constexpr int kWarps = kSolveThreads / 32;

template <typename T>
struct ChainDev {
  const int32_t *first, *n, *m, *parent, *child, *uidx, *rel, *ldn, *ldm;
  const int32_t* ginv;      // inverse extend-add maps, 2 x (n + m) per supernode
  const int64_t* ginv_off;
  const int32_t *nch_f, *nch_b, *level;
  int sub_front;  // per-warp vector capacity for subtree tasks
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
  const int* set_of;  // factor set of each solve slot
  int n_bins;
  int B, tau0, tau1, trans;
  int Borb;  // multi-RHS kernel: right-hand sides in the launch (B counts their groups)
  int total;
  long long spin_limit;
  int never_ready;  // self-test: the first task waits for a count nothing reaches
  int prefetch;     // L2 prefetch of each task's factor rows before its dependency wait
  int stream_ef;    // factor rows read once per launch: evict-first loads
  int64_t prefetch_bytes;  // at most this many bytes of a task's rows are prefetched
  unsigned spin_ns;  // longest sleep between polls of a completion counter
  int ngroups;  // task groups (orbits or right-hand-side groups) split into ngroups ...
  int goff;     // ... whose phase sequences start goff phases apart
};

// Claim order.  A launch's work is nb bins x nphase phases (fwd leaves->root,
// bwd root->leaves) for B task groups (single orbits, or groups of
// right-hand sides).  The groups are split into D.ngroups sets; set gr runs its
// global phase g = bin * nphase + phase at slot g + gr * D.goff, and tasks are
// claimed slot by slot (set, then group, then item within a slot).  With one
// set this is the plain bin / phase / group order; with several, the sets reach
// the few large tasks at the top of the tree at different times, so tasks of
// the other sets fill the GPU meanwhile.  Every dependency lies inside one
// group (earlier phase or bin of the same orbit), so it is still claimed
// earlier, and the earliest unfinished task can always run.
constexpr int kMaxSlots = 9 * kMaxPhases + 1;
constexpr int kMaxSets = 8;

// Shared tables of the claim order: first task of every slot, first group of
// every set, task count of every phase.
struct SlotTables {
  int slot[kMaxSlots];
  int set_first[kMaxSets + 1];
  int cnt[kMaxPhases];
  int nslot, G;
};

template <typename T>
__device__ __forceinline__ void build_slots(const ChainDev<T>& D, SlotTables& S) {
  const int nb = D.total / (D.items_per_bin * D.B);
  const int G = nb * D.nphase;
  const int nslot = G + (D.ngroups - 1) * D.goff;
  for (int i = threadIdx.x; i < D.nphase; i += blockDim.x) S.cnt[i] = D.phase_off[i + 1] - D.phase_off[i];
  for (int i = threadIdx.x; i <= D.ngroups; i += blockDim.x) S.set_first[i] = (int)(((int64_t)i * D.B) / D.ngroups);
  __syncthreads();
  for (int sg = threadIdx.x; sg < nslot; sg += blockDim.x) {
    int sz = 0;
    for (int gr = 0; gr < D.ngroups; ++gr) {
      const int g = sg - gr * D.goff;
      if (g >= 0 && g < G) sz += S.cnt[g % D.nphase] * (S.set_first[gr + 1] - S.set_first[gr]);
    }
    S.slot[sg + 1] = sz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    S.slot[0] = 0;
    for (int sg = 1; sg <= nslot; ++sg) S.slot[sg] += S.slot[sg - 1];
    S.nslot = nslot;
    S.G = G;
  }
  __syncthreads();
}

// Task t -> bin q (0-based in the launch), phase p, group index gi, item index.
template <typename T>
__device__ __forceinline__ void decode_task(const ChainDev<T>& D, const SlotTables& S, int t, int& q, int& p,
                                            int& gi, int& item) {
  int lo = 0, hi = S.nslot;  // slot with slot[lo] <= t < slot[lo + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (S.slot[mid] <= t) lo = mid;
    else hi = mid;
  }
  int rem = t - S.slot[lo];
  for (int gr = 0; gr < D.ngroups; ++gr) {
    const int g = lo - gr * D.goff;
    if (g < 0 || g >= S.G) continue;
    const int pp = g % D.nphase;
    const int cnt = S.cnt[pp];
    const int sz = cnt * (S.set_first[gr + 1] - S.set_first[gr]);
    if (rem < sz) {
      const int k = rem / cnt;
      q = g / D.nphase;
      p = pp;
      gi = S.set_first[gr] + k;
      item = D.phase_off[pp] + (rem - k * cnt);
      return;
    }
    rem -= sz;
  }
  q = p = gi = item = 0;  // not reached for t < total
}

// Bounded spin on a completion counter: sleeps between polls double from
// 32 ns up to max_ns; `limit` polls at most, then ORBIT_ERR_TIMEOUT.
__device__ __forceinline__ bool wait_ge(const int* p, int target, int* status, long long limit,
                                        unsigned max_ns = 1024) {
  long long it = 0;
  unsigned ns = 32;
  while (ld_acquire(p) < target) {
    if (ld_volatile(status) != 0) return false;
    if (++it > limit) {
      raise_status(status, ORBIT_ERR_TIMEOUT);
      return false;
    }
    __nanosleep(ns);
    if (ns < max_ns) ns <<= 1;
  }
  return true;
}

// Vector types for 16-byte loads of factor rows (rows start 16-byte aligned:
// every leading dimension and block offset is a multiple of 4 elements).
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int w = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int w = 2; };

__device__ __forceinline__ float dot16(const float4& a, const float* v) {
  return a.x * v[0] + a.y * v[1] + a.z * v[2] + a.w * v[3];
}
__device__ __forceinline__ double dot16(const double2& a, const double* v) {
  return a.x * v[0] + a.y * v[1];
}

// 16-byte loads in flight per lane in the row dot products of the chained
// solves, per precision.  Measured on the 80x72x15 grid (8 bins, CUDA events):
// FP32, 12 orbits at 10 CTAs per SM: 7.21 ms at 4, 6.94 at 6, 7.05 at 7 (8 at
// 8 CTAs per SM: 7.55); FP64 at 7 CTAs per SM, 1 / 12 orbits: 1.76 / 9.83 ms
// at 12 (2.44 ms / - at 4 and 8 CTAs per SM; 1.81 / 10.9 at 10; 1.81 / 11.1
// at 16 and 6 CTAs per SM).
#ifndef ORBIT_SOLVE_DEPTH_FP32
#define ORBIT_SOLVE_DEPTH_FP32 6
#endif
#ifndef ORBIT_SOLVE_DEPTH_FP64
#define ORBIT_SOLVE_DEPTH_FP64 12
#endif
template <typename T> struct Depth { static constexpr int value = sizeof(T) == 4 ? ORBIT_SOLVE_DEPTH_FP32 : ORBIT_SOLVE_DEPTH_FP64; };

// Factor rows that a launch reads once (every solve slot has its own factor
// set) are loaded under an L2 evict-first policy, so that they do not push out
// the lines the tasks' prefetches brought in, nor the solution vectors; where
// slots share a set the rows are reused from L2 and load under the normal
// policy (the many-right-hand-side kernel keeps plain loads).  Measured on the
// 80x72x15 grid (8 bins, CUDA events): the 12-orbit FP32 chain 6.44-6.50 ms
// with evict-first against 6.58-6.62 without a hint, 6.54 with no L1
// allocation (alone or with evict-first), 6.57 with evict-last prefetches;
// the single-orbit FP64 chain unchanged (1.72 ms); evict-first in the 64-RHS
// kernels, where the groups share one set: 24.6 vs 20.9 ms transposed and
// 22.0 vs 20.7 ms forward.
__device__ __forceinline__ uint64_t stream_policy(bool evict_first) {
  uint64_t pol;
  if (evict_first) asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  else asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

__device__ __forceinline__ float4 ld_stream(const float4* p, uint64_t pol) {
  float4 x;
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w) : "l"(p), "l"(pol));
  return x;
}

__device__ __forceinline__ double2 ld_stream(const double2* p, uint64_t pol) {
  double2 x;
  asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(x.x), "=d"(x.y) : "l"(p), "l"(pol));
  return x;
}

// Per-lane partial of sum_{j0 <= j < j1} a[j] v[j] for a group of G lanes
// (gl = lane within the group; a 16-byte aligned at j = 0, v in shared memory,
// 16-byte aligned).  16-byte loads, up to U in flight per lane: the unrolled
// loop issues its guarded loads before it uses any of them.
template <typename T, int G = 32, int U = Depth<T>::value>
__device__ __forceinline__ T dot_seg(const T* __restrict__ a, const T* v, int j0, int j1, int gl, uint64_t pol) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::w;
  T acc0 = T(0), acc1 = T(0), acc2 = T(0), acc3 = T(0);
  // [j0, ja) scalar head up to the first aligned index, [ja, jb) 16-byte
  // vectors, [jb, j1) scalar tail
  const int ja = min((j0 + W - 1) / W * W, j1);
  const int jb = max(ja, j1 / W * W);
  for (int j = j0 + gl; j < ja; j += G) acc0 = fma(__ldg(a + j), v[j], acc0);
  const int nv0 = ja / W, nv1 = jb / W;
  const V* a4 = reinterpret_cast<const V*>(a);
  for (int k = nv0 + gl; k < nv1; k += U * G) {
    V x[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      x[u] = V{};
      if (u == 0 || k + u * G < nv1) x[u] = ld_stream(a4 + k + u * G, pol);
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (u == 0 || k + u * G < nv1) {
        const T d = dot16(x[u], v + (k + u * G) * W);
        if ((u & 3) == 0) acc0 += d;
        else if ((u & 3) == 1) acc1 += d;
        else if ((u & 3) == 2) acc2 += d;
        else acc3 += d;
      }
  }
  for (int j = jb + gl; j < j1; j += G) acc1 = fma(__ldg(a + j), v[j], acc1);
  return (acc0 + acc1) + (acc2 + acc3);
}

// Rows [r0, r1) of a row-major block as dot products, G lanes per row, so a
// warp works on 32 / G rows at once; warps wid, wid + nw, ... of the caller
// take successive row groups.  partial(g, i, gl) is a lane's share of row i
// (g is G as a std::integral_constant, for the matching dot_seg stride);
// store(i, sum) runs on the group's first lane.  The trip count is uniform
// across the warp (the shuffles are warp-wide).
template <int G, typename T, typename P, typename S>
__device__ __forceinline__ void grouped_rows(int r0, int r1, int wid, int nw, P&& partial, S&& store) {
  constexpr int R = 32 / G;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gr = lane / G;
  for (int i0 = r0 + wid * R; i0 < r1; i0 += nw * R) {
    const int i = i0 + gr;
    T acc = i < r1 ? partial(std::integral_constant<int, G>(), i, gl) : T(0);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (i < r1 && gl == 0) store(i, acc);
  }
}

// Lanes per row from the longest row of the range: about U 16-byte vectors
// per lane (U loads in flight), between 4 and 32 lanes.
template <typename T, int U = 4>
__device__ __forceinline__ int group_lanes(int maxlen) {
  const int nv = (maxlen + Vec16<T>::w - 1) / Vec16<T>::w;
  return nv <= 4 * U ? 4 : nv <= 8 * U ? 8 : nv <= 16 * U ? 16 : 32;
}

#define ORBIT_GROUPED_ROWS(T, G_, r0, r1, wid, nw, partial, store)           \
  do {                                                                      \
    switch (G_) {                                                           \
      case 4: grouped_rows<4, T>(r0, r1, wid, nw, partial, store); break;   \
      case 8: grouped_rows<8, T>(r0, r1, wid, nw, partial, store); break;   \
      case 16: grouped_rows<16, T>(r0, r1, wid, nw, partial, store); break; \
      default: grouped_rows<32, T>(r0, r1, wid, nw, partial, store); break; \
    }                                                                       \
  } while (0)

// Column-oriented partial dot products of the transposed sweeps: this warp's
// share (rows i0 + warp, i0 + warp + kWarps, ... below i1) of
// sum_i a[i * stride] v_k[i] for nk <= K vectors v_k = v + k * vcap, with
// four loads in flight (lanes hold consecutive columns, so every row step is
// one coalesced 128-byte read per warp).
template <typename T, int K>
__device__ __forceinline__ void col_dot(const T* __restrict__ a, int64_t stride, int i0, int i1, const T* v,
                                        int vcap, int nk, T (&acc)[K]) {
  int i = i0 + (threadIdx.x >> 5);
  for (; i + 3 * kWarps < i1; i += 4 * kWarps) {
    const T x0 = __ldg(a + (int64_t)i * stride);
    const T x1 = __ldg(a + (int64_t)(i + kWarps) * stride);
    const T x2 = __ldg(a + (int64_t)(i + 2 * kWarps) * stride);
    const T x3 = __ldg(a + (int64_t)(i + 3 * kWarps) * stride);
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < nk) {
        const T* vk = v + k * vcap;
        acc[k] = fma(x0, vk[i], acc[k]);
        acc[k] = fma(x1, vk[i + kWarps], acc[k]);
        acc[k] = fma(x2, vk[i + 2 * kWarps], acc[k]);
        acc[k] = fma(x3, vk[i + 3 * kWarps], acc[k]);
      }
  }
  for (; i < i1; i += kWarps) {
    const T x = __ldg(a + (int64_t)i * stride);
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < nk) acc[k] = fma(x, v[k * vcap + i], acc[k]);
  }
}

// Forward step of one supernode (L, or U^T when trans) for output rows
// [r0, r1): gathers its right-hand side (own entries of Xin, plus forcing) and
// the children's update vectors into `vec`, then one dense GEMV.  Ends with a
// block barrier.
template <typename T>
__device__ __forceinline__ void fwd_node(const ChainDev<T>& D, int o, int tau, int s, int r0, int r1, bool trans,
                                         T* vec, T* red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t N = D.N;
  const int n = D.n[s], m = D.m[s], first = D.first[s];
  const int ldn = D.ldn[s], ldm = D.ldm[s];
  const T* SQ = D.factors + ((int64_t)D.set_of[o] * D.n_bins + tau) * D.fac_size + D.fac_off[s];
  const uint64_t pol = stream_policy(D.stream_ef != 0);
  double* Yo = D.Y + (int64_t)o * N;
  double* Wo = D.W + (int64_t)o * D.w_size;
  const int bin_in = trans ? tau + 1 : tau;
  const double* Xin = D.X + ((int64_t)o * 9 + bin_in) * N;
  const double* Ein = nullptr;
  if (D.E) {
    if (!trans) Ein = D.E + ((int64_t)o * 8 + tau) * N;
    else if (tau + 1 < D.tau1) Ein = D.E + ((int64_t)o * 8 + tau + 1) * N;
  }
  // Rows (or columns) [r0, r1) read vec on [0, min(r1, n)) and on
  // [max(r0, n), r1): only that part is gathered, in one pass, each position
  // pulling its own entry and the children's update entries that land on it
  // (inverse extend-add maps, -1 where a child contributes nothing).
  const int lo_end = min(r1, n), hi0 = max(r0, n);
  const int w = n + m;
  const int32_t* g0 = D.ginv + D.ginv_off[s];
  const int32_t* g1 = g0 + w;
  const int c0 = D.child[2 * s], c1 = D.child[2 * s + 1];
  const double* W0 = c0 >= 0 ? Wo + D.woff[c0] : nullptr;
  const double* W1 = c1 >= 0 ? Wo + D.woff[c1] : nullptr;
  for (int i = tid; i < lo_end; i += kSolveThreads) {
    double v = Xin[first + i];
    if (Ein) v += D.escale * Ein[first + i];
    const int u0 = g0[i], u1 = g1[i];
    if (u0 >= 0) v += W0[u0];
    if (u1 >= 0) v += W1[u1];
    vec[i] = (T)v;
  }
  for (int i = hi0 + tid; i < r1; i += kSolveThreads) {
    double v = 0.0;
    const int u0 = g0[i], u1 = g1[i];
    if (u0 >= 0) v += W0[u0];
    if (u1 >= 0) v += W1[u1];
    vec[i] = (T)v;
  }
  __syncthreads();
  if (!trans) {
    // rows of [SQ; Pb]: row i < n uses the strict lower part (unit diagonal)
    const int64_t woff = D.woff[s];
    auto partial = [&](auto g, int i, int gl) {
      return dot_seg<T, decltype(g)::value>(SQ + (int64_t)i * ldn, vec, 0, i < n ? i : n, gl, pol);
    };
    auto store = [&](int i, T acc) {
      if (i < n) Yo[first + i] = (double)(vec[i] + acc);
      else Wo[woff + (i - n)] = (double)(vec[i] + acc);
    };
    const int G = group_lanes<T, Depth<T>::value>(min(r1 - 1, n));
    ORBIT_GROUPED_ROWS(T, G, r0, r1, warp, kWarps, partial, store);
  } else {
    // columns of [upper(SQ) | Qr]
    const T* Qr = SQ + (int64_t)(n + m) * ldn;
    for (int cb = r0; cb < r1; cb += 32) {
      const int c = cb + lane;
      T a1[1] = {T(0)};
      if (c < r1) {
        if (c < n) col_dot<T, 1>(SQ + c, ldn, 0, c + 1, vec, 0, 1, a1);
        else col_dot<T, 1>(Qr + (c - n), ldm, 0, n, vec, 0, 1, a1);
      }
      const T acc = a1[0];
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
// own forward result plus the ancestors' solution; the ancestor part of `vec`
// starts at the next 4-element boundary after the own part so both segments
// can be read with 16-byte loads.  Ends with a block barrier.
template <typename T>
__device__ __forceinline__ void bwd_node(const ChainDev<T>& D, int o, int tau, int s, int r0, int r1, bool trans,
                                         T* vec, T* red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t N = D.N;
  const int n = D.n[s], m = D.m[s], first = D.first[s];
  const int ldn = D.ldn[s], ldm = D.ldm[s];
  const int n0pad = (n + 3) & ~3;
  const T* SQ = D.factors + ((int64_t)D.set_of[o] * D.n_bins + tau) * D.fac_size + D.fac_off[s];
  const uint64_t pol = stream_policy(D.stream_ef != 0);
  const double* Yo = D.Y + (int64_t)o * N;
  const int bin_out = trans ? tau : tau + 1;
  double* Xout = D.X + ((int64_t)o * 9 + bin_out) * N;
  const int32_t* ui = D.uidx + D.uoff[s];
  // rows (or columns) [r0, r1) read the own part of vec from r0 on
  for (int i = r0 + tid; i < n; i += kSolveThreads) vec[i] = (T)Yo[first + i];
  for (int u = tid; u < m; u += kSolveThreads) vec[n0pad + u] = (T)Xout[ui[u]];
  __syncthreads();
  if (!trans) {
    const T* Qr = SQ + (int64_t)(n + m) * ldn;
    auto partial = [&](auto g, int i, int gl) {
      constexpr int G = decltype(g)::value;
      return dot_seg<T, G>(SQ + (int64_t)i * ldn, vec, i, n, gl, pol) +
             dot_seg<T, G>(Qr + (int64_t)i * ldm, vec + n0pad, 0, m, gl, pol);
    };
    auto store = [&](int i, T acc) { Xout[first + i] = (double)acc; };
    const int G = group_lanes<T, Depth<T>::value>(n - r0 + m);
    ORBIT_GROUPED_ROWS(T, G, r0, r1, warp, kWarps, partial, store);
  } else {
    // columns of [SQ_strict_lower ; Pb] with unit diagonal
    const T* Pb = SQ + (int64_t)n * ldn;
    for (int cb = r0; cb < r1; cb += 32) {
      const int c = cb + lane;
      T a1[1] = {T(0)};
      if (c < r1) {
        col_dot<T, 1>(SQ + c, ldn, c + 1, n, vec, 0, 1, a1);
        col_dot<T, 1>(Pb + c, ldn, 0, m, vec + n0pad, 0, 1, a1);
      }
      const T acc = a1[0];
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

// Warp-level forward step of one small supernode (inside a subtree task).
template <typename T>
__device__ void fwd_node_warp(const ChainDev<T>& D, int o, int tau, int s, bool trans, T* v) {
  const int lane = threadIdx.x & 31;
  const int64_t N = D.N;
  const int n = D.n[s], m = D.m[s], first = D.first[s];
  const int ldn = D.ldn[s], ldm = D.ldm[s];
  const T* SQ = D.factors + ((int64_t)D.set_of[o] * D.n_bins + tau) * D.fac_size + D.fac_off[s];
  const uint64_t pol = stream_policy(D.stream_ef != 0);
  double* Yo = D.Y + (int64_t)o * N;
  double* Wo = D.W + (int64_t)o * D.w_size;
  const int bin_in = trans ? tau + 1 : tau;
  const double* Xin = D.X + ((int64_t)o * 9 + bin_in) * N;
  const double* Ein = nullptr;
  if (D.E) {
    if (!trans) Ein = D.E + ((int64_t)o * 8 + tau) * N;
    else if (tau + 1 < D.tau1) Ein = D.E + ((int64_t)o * 8 + tau + 1) * N;
  }
  for (int i = lane; i < n + m; i += 32) {
    double x = 0.0;
    if (i < n) {
      x = Xin[first + i];
      if (Ein) x += D.escale * Ein[first + i];
    }
    v[i] = (T)x;
  }
  for (int q2 = 0; q2 < 2; ++q2) {
    __syncwarp();
    const int c = D.child[2 * s + q2];
    if (c < 0) continue;
    const int mc = D.m[c];
    const int32_t* rel = D.rel + D.uoff[c];
    const double* wc = Wo + D.woff[c];
    for (int j = lane; j < mc; j += 32) v[rel[j]] += (T)wc[j];
  }
  __syncwarp();
  const int64_t woff = D.woff[s];
  if (!trans) {
    if (n <= 64) {
      for (int i = lane; i < n + m; i += 32) {
        const int len = i < n ? i : n;
        const T* row = SQ + (int64_t)i * ldn;
        T acc = T(0);
        for (int j = 0; j < len; ++j) acc = fma(__ldg(row + j), v[j], acc);
        if (i < n) Yo[first + i] = (double)(v[i] + acc);
        else Wo[woff + (i - n)] = (double)(v[i] + acc);
      }
    } else {
      auto partial = [&](auto g, int i, int gl) {
        return dot_seg<T, decltype(g)::value>(SQ + (int64_t)i * ldn, v, 0, i < n ? i : n, gl, pol);
      };
      auto store = [&](int i, T acc) {
        if (i < n) Yo[first + i] = (double)(v[i] + acc);
        else Wo[woff + (i - n)] = (double)(v[i] + acc);
      };
      const int G = group_lanes<T>(n);
      ORBIT_GROUPED_ROWS(T, G, 0, n + m, 0, 1, partial, store);
    }
  } else {
    const T* Qr = SQ + (int64_t)(n + m) * ldn;
    for (int c = lane; c < n + m; c += 32) {
      T acc = T(0);
      if (c < n) {
        for (int i = 0; i <= c; ++i) acc = fma(__ldg(SQ + (int64_t)i * ldn + c), v[i], acc);
        Yo[first + c] = (double)acc;
      } else {
        const int u = c - n;
        for (int i = 0; i < n; ++i) acc = fma(__ldg(Qr + (int64_t)i * ldm + u), v[i], acc);
        Wo[woff + u] = (double)(v[c] + acc);
      }
    }
  }
  __syncwarp();
}

// Warp-level backward step of one small supernode (inside a subtree task).
template <typename T>
__device__ void bwd_node_warp(const ChainDev<T>& D, int o, int tau, int s, bool trans, T* v) {
  const int lane = threadIdx.x & 31;
  const int64_t N = D.N;
  const int n = D.n[s], m = D.m[s], first = D.first[s];
  const int ldn = D.ldn[s], ldm = D.ldm[s];
  const int n0pad = (n + 3) & ~3;
  const T* SQ = D.factors + ((int64_t)D.set_of[o] * D.n_bins + tau) * D.fac_size + D.fac_off[s];
  const uint64_t pol = stream_policy(D.stream_ef != 0);
  const double* Yo = D.Y + (int64_t)o * N;
  const int bin_out = trans ? tau : tau + 1;
  double* Xout = D.X + ((int64_t)o * 9 + bin_out) * N;
  const int32_t* ui = D.uidx + D.uoff[s];
  for (int i = lane; i < n; i += 32) v[i] = (T)Yo[first + i];
  for (int u = lane; u < m; u += 32) v[n0pad + u] = (T)Xout[ui[u]];
  __syncwarp();
  if (!trans) {
    const T* Qr = SQ + (int64_t)(n + m) * ldn;
    auto partial = [&](auto g, int i, int gl) {
      constexpr int G = decltype(g)::value;
      return dot_seg<T, G>(SQ + (int64_t)i * ldn, v, i, n, gl, pol) +
             dot_seg<T, G>(Qr + (int64_t)i * ldm, v + n0pad, 0, m, gl, pol);
    };
    auto store = [&](int i, T acc) { Xout[first + i] = (double)acc; };
    const int G = group_lanes<T>(n + m);
    ORBIT_GROUPED_ROWS(T, G, 0, n, 0, 1, partial, store);
  } else {
    const T* Pb = SQ + (int64_t)n * ldn;
    for (int c = lane; c < n; c += 32) {
      T acc = v[c];
      for (int i = c + 1; i < n; ++i) acc = fma(__ldg(SQ + (int64_t)i * ldn + c), v[i], acc);
      for (int u = 0; u < m; ++u) acc = fma(__ldg(Pb + (int64_t)u * ldn + c), v[n0pad + u], acc);
      Xout[first + c] = (double)acc;
    }
  }
  __syncwarp();
}

// One instantiation per sweep direction (TR: transposed) and per schedule
// kind (SUB: the schedule has whole-subtree tasks), so that each kernel
// carries only the code its tasks run.
template <typename T, bool TR, bool SUB>
__global__ void __launch_bounds__(kSolveThreads, sizeof(T) == 4 ? ORBIT_SOLVE_MINB_FP32 : ORBIT_SOLVE_MINB) k_chain(ChainDev<T> D) {
  extern __shared__ unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);      // kWarps * 32
  T* vec = red + kWarps * 32;                    // front-sized vector
  __shared__ int s_task;
  __shared__ int s_ok;   // status word clean at the claim
  __shared__ int s_dep;  // dependency wait succeeded
  __shared__ SlotTables s_tab;
  const int tid = threadIdx.x;
  build_slots(D, s_tab);
  for (;;) {
    if (tid == 0) {
      s_task = atomicAdd(D.task_counter, 1);
      s_ok = ld_volatile(D.status) == 0;
    }
    __syncthreads();
    const int t = s_task;
    if (t >= D.total || !s_ok) break;
    int q, p, oi, item;
    decode_task(D, s_tab, t, q, p, oi, item);
    const int tau = TR ? (D.tau1 - 1 - q) : (D.tau0 + q);
    const int4 it = D.items[item];
    const int o = D.orbit_ids[oi];
    const int s = it.x, kind = it.w;
    const bool fwd = (kind & 1) == 0;        // kinds 0, 2, 4, 6
    const bool trans = TR;                   // kinds 2, 3, 6, 7
    const bool subtree = SUB && kind >= 4;
    int* cbase = D.counters + (int64_t)o * 8 * 2 * D.nsuper;
    // The factor rows of a row-chunk task do not depend on other tasks: ask L2
    // for them before waiting (forward: whole rows of [SQ; Pb]; backward: the
    // upper part of the SQ rows and the Qr rows), one request per 128 bytes.
    // Off for FP64 at large batches, where the launch is throughput-bound and
    // the requests only cost issue slots.
    if (D.prefetch && (kind == 0 || kind == 1)) {
      const int n_s = D.n[s], ldn_s = D.ldn[s];
      const T* SQ = D.factors + ((int64_t)D.set_of[o] * D.n_bins + tau) * D.fac_size + D.fac_off[s];
      constexpr int L = 128 / sizeof(T);
      if (kind == 0) {
        const char* a = reinterpret_cast<const char*>(SQ + (int64_t)it.y * ldn_s);
        const int64_t bytes = min((int64_t)(it.z - it.y) * ldn_s * (int64_t)sizeof(T), D.prefetch_bytes);
        for (int64_t q = (int64_t)tid * 128; q < bytes; q += (int64_t)kSolveThreads * 128)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a + q));
      } else {
        const int ldm_s = D.ldm[s], m_s = D.m[s];
        const T* Qr = SQ + (int64_t)(n_s + m_s) * ldn_s;
        const int64_t row_bytes = (int64_t)(n_s + m_s) * sizeof(T);
        const int i_end = (int)min((int64_t)it.z, it.y + max((int64_t)1, D.prefetch_bytes / row_bytes));
        for (int i = it.y + (tid >> 3); i < i_end; i += kSolveThreads / 8) {
          const T* row = SQ + (int64_t)i * ldn_s;
          for (int c = (i & ~(L - 1)) + (tid & 7) * L; c < n_s; c += 8 * L)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(row + c));
          const T* qrow = Qr + (int64_t)i * ldm_s;
          for (int c = (tid & 7) * L; c < m_s; c += 8 * L) asm volatile("prefetch.global.L2 [%0];" ::"l"(qrow + c));
        }
      }
    }
    // ---- dependencies ----
    if (tid == 0) {
      bool ok = true;
      if (D.never_ready && t == 0)
        ok = wait_ge(cbase + (tau * 2 + 0) * D.nsuper + s, 0x7fffffff, D.status, D.spin_limit, D.spin_ns);
      if (!ok) {
      } else if (fwd) {
        if (!subtree)
          for (int q2 = 0; q2 < 2 && ok; ++q2) {
            const int c = D.child[2 * s + q2];
            if (c >= 0) ok = wait_ge(cbase + (tau * 2 + 0) * D.nsuper + c, D.nch_f[c], D.status, D.spin_limit, D.spin_ns);
          }
        if (ok && !trans && tau > D.tau0)
          ok = wait_ge(cbase + ((tau - 1) * 2 + 1) * D.nsuper + s, D.nch_b[s], D.status, D.spin_limit, D.spin_ns);
        if (ok && trans && tau < D.tau1 - 1)
          ok = wait_ge(cbase + ((tau + 1) * 2 + 1) * D.nsuper + s, D.nch_b[s], D.status, D.spin_limit, D.spin_ns);
      } else {
        const int par = D.parent[s];
        if (par < 0)
          ok = wait_ge(cbase + (tau * 2 + 0) * D.nsuper + s, D.nch_f[s], D.status, D.spin_limit, D.spin_ns);
        else
          ok = wait_ge(cbase + (tau * 2 + 1) * D.nsuper + par, D.nch_b[par], D.status, D.spin_limit, D.spin_ns);
      }
      s_dep = ok;
    }
    __syncthreads();
    if (!s_dep) break;
    if (!subtree) {
      if (fwd) fwd_node(D, o, tau, s, it.y, it.z, trans, vec, red);
      else bwd_node(D, o, tau, s, it.y, it.z, trans, vec, red);
    } else {
      // Whole subtree in this CTA: depth by depth (deepest first for the
      // forward sweep, root first for the backward sweep), the supernodes of
      // one depth spread over the warps, one warp per supernode.
      const int warp = threadIdx.x >> 5;
      T* wv = vec + warp * ((D.sub_front + 7) & ~3);
      const int d0 = it.y;
      const int top = D.level[s];
      int deep = top;
      for (int d = d0; d <= s; ++d) deep = max(deep, D.level[d]);
      for (int q3 = 0; q3 <= deep - top; ++q3) {
        const int lev = fwd ? deep - q3 : top + q3;
        int k = 0;
        for (int d = d0; d <= s; ++d) {
          if (D.level[d] != lev) continue;
          if ((k++ & (kWarps - 1)) != warp) continue;
          if (fwd) fwd_node_warp(D, o, tau, d, trans, wv);
          else bwd_node_warp(D, o, tau, d, trans, wv);
        }
        __syncthreads();
      }
    }
    if (tid == 0) {
      red_release_add(cbase + (tau * 2 + (fwd ? 0 : 1)) * D.nsuper + s, 1);
    }
  }
}

// ---- many right-hand sides on one factor set ----
//
// When every solve slot of a handle maps onto the same factor set (marginal
// perturbations or adjoint receptors of one operator), each task serves a
// group of K right-hand sides: one claim, one dependency wait (on the group's
// counters) and one barrier sequence, and every factor row loaded once is
// multiplied against the K gathered vectors.  Non-transposed sweeps only.

template <typename T, int G, int K>
__device__ __forceinline__ void dot_seg_multi(const T* __restrict__ a, const T* v, int vcap, int nk, int j0, int j1,
                                              int gl, T (&acc)[K]) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::w;
  const int ja = min((j0 + W - 1) / W * W, j1);
  const int jb = max(ja, j1 / W * W);
  for (int j = j0 + gl; j < ja; j += G) {
    const T x = __ldg(a + j);
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < nk) acc[k] = fma(x, v[k * vcap + j], acc[k]);
  }
  const V* a4 = reinterpret_cast<const V*>(a);
  const int nv0 = ja / W, nv1 = jb / W;
  for (int kk = nv0 + gl; kk < nv1; kk += 2 * G) {
    const bool b1 = kk + G < nv1;
    V x1 = {};
    const V x0 = __ldg(a4 + kk);
    if (b1) x1 = __ldg(a4 + kk + G);
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < nk) {
        acc[k] += dot16(x0, v + k * vcap + kk * W);
        if (b1) acc[k] += dot16(x1, v + k * vcap + (kk + G) * W);
      }
  }
  for (int j = jb + gl; j < j1; j += G) {
    const T x = __ldg(a + j);
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < nk) acc[k] = fma(x, v[k * vcap + j], acc[k]);
  }
}

template <int G, int K, typename T, typename P, typename S>
__device__ __forceinline__ void grouped_rows_multi(int r0, int r1, int wid, int nw, P&& partial, S&& store) {
  constexpr int R = 32 / G;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gr = lane / G;
  for (int i0 = r0 + wid * R; i0 < r1; i0 += nw * R) {
    const int i = i0 + gr;
    T acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = T(0);
    if (i < r1) partial(std::integral_constant<int, G>(), i, gl, acc);
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (i < r1 && gl == 0) store(i, acc);
  }
}

#define ORBIT_GROUPED_ROWS_MULTI(T, K, G_, r0, r1, wid, nw, partial, store)            \
  do {                                                                                \
    switch (G_) {                                                                     \
      case 4: grouped_rows_multi<4, K, T>(r0, r1, wid, nw, partial, store); break;    \
      case 8: grouped_rows_multi<8, K, T>(r0, r1, wid, nw, partial, store); break;    \
      case 16: grouped_rows_multi<16, K, T>(r0, r1, wid, nw, partial, store); break;  \
      default: grouped_rows_multi<32, K, T>(r0, r1, wid, nw, partial, store); break;  \
    }                                                                                 \
  } while (0)

template <typename T, int K>
__global__ void __launch_bounds__(kSolveThreads, sizeof(T) == 4 ? ORBIT_SOLVE_MINB_FP32 : ORBIT_SOLVE_MINB) k_chain_multi(ChainDev<T> D, int vcap) {
  extern __shared__ unsigned char smem_raw[];
  T* vbuf = reinterpret_cast<T*>(smem_raw);  // K vectors of vcap
  T* red = vbuf + (int64_t)K * vcap;          // K x kWarps x 32 (transposed sweeps)
  __shared__ int s_task;
  __shared__ int s_ok;   // status word clean at the claim
  __shared__ int s_dep;  // dependency wait succeeded
  __shared__ SlotTables s_tab;
  const int tid = threadIdx.x, warp = tid >> 5;
  build_slots(D, s_tab);
  for (;;) {
    if (tid == 0) {
      s_task = atomicAdd(D.task_counter, 1);
      s_ok = ld_volatile(D.status) == 0;
    }
    __syncthreads();
    const int t = s_task;
    if (t >= D.total || !s_ok) break;
    int q, pph, gi, item;
    decode_task(D, s_tab, t, q, pph, gi, item);
    const int tau = D.trans ? (D.tau1 - 1 - q) : (D.tau0 + q);
    const int4 it = D.items[item];
    const int s = it.x, kind = it.w, r0 = it.y, r1 = it.z;
    const int nk = min(K, D.Borb - gi * K);
    int o[K];
#pragma unroll
    for (int k = 0; k < K; ++k) o[k] = D.orbit_ids[gi * K + (k < nk ? k : 0)];
    int* cbase = D.counters + (int64_t)o[0] * 8 * 2 * D.nsuper;  // the group's counters
    const int n = D.n[s], m = D.m[s], first = D.first[s], ldn = D.ldn[s], ldm = D.ldm[s];
    const T* SQ = D.factors + ((int64_t)D.set_of[o[0]] * D.n_bins + tau) * D.fac_size + D.fac_off[s];
    if (D.prefetch) {
      if (kind == 0) {
        const char* a = reinterpret_cast<const char*>(SQ + (int64_t)r0 * ldn);
        const int64_t bytes = min((int64_t)(r1 - r0) * ldn * (int64_t)sizeof(T), D.prefetch_bytes);
        for (int64_t q2 = (int64_t)tid * 128; q2 < bytes; q2 += (int64_t)kSolveThreads * 128)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a + q2));
      }
    }
    if (tid == 0) {
      bool ok = true;
      if (kind == 0 || kind == 2) {
        for (int q2 = 0; q2 < 2 && ok; ++q2) {
          const int c = D.child[2 * s + q2];
          if (c >= 0) ok = wait_ge(cbase + (tau * 2 + 0) * D.nsuper + c, D.nch_f[c], D.status, D.spin_limit, D.spin_ns);
        }
        if (ok && kind == 0 && tau > D.tau0)
          ok = wait_ge(cbase + ((tau - 1) * 2 + 1) * D.nsuper + s, D.nch_b[s], D.status, D.spin_limit, D.spin_ns);
        if (ok && kind == 2 && tau < D.tau1 - 1)
          ok = wait_ge(cbase + ((tau + 1) * 2 + 1) * D.nsuper + s, D.nch_b[s], D.status, D.spin_limit, D.spin_ns);
      } else {
        const int par = D.parent[s];
        if (par < 0) ok = wait_ge(cbase + (tau * 2 + 0) * D.nsuper + s, D.nch_f[s], D.status, D.spin_limit, D.spin_ns);
        else ok = wait_ge(cbase + (tau * 2 + 1) * D.nsuper + par, D.nch_b[par], D.status, D.spin_limit, D.spin_ns);
      }
      s_dep = ok;
    }
    __syncthreads();
    if (!s_dep) break;
    const int n0pad = (n + 3) & ~3;
    const int lane = tid & 31;
    if (kind == 2) {
      // transposed forward (U^T, then the update columns): gather over
      // [0, min(r1, n)) and [max(r0, n), r1) as the forward rows do, then
      // columns [r0, r1) of [upper(SQ) | Qr], each factor element used for
      // the K vectors
      const int lo_end = min(r1, n), hi0 = max(r0, n), w = n + m;
      const int32_t* g0 = D.ginv + D.ginv_off[s];
      const int32_t* g1 = g0 + w;
      const int c0 = D.child[2 * s], c1 = D.child[2 * s + 1];
      for (int k = 0; k < nk; ++k) {
        T* vec = vbuf + k * vcap;
        const double* Xin = D.X + ((int64_t)o[k] * 9 + tau + 1) * D.N;
        const double* Ein = (D.E && tau + 1 < D.tau1) ? D.E + ((int64_t)o[k] * 8 + tau + 1) * D.N : nullptr;
        const double* Wo = D.W + (int64_t)o[k] * D.w_size;
        const double* W0 = c0 >= 0 ? Wo + D.woff[c0] : nullptr;
        const double* W1 = c1 >= 0 ? Wo + D.woff[c1] : nullptr;
        for (int i = tid; i < lo_end; i += kSolveThreads) {
          double v = Xin[first + i];
          if (Ein) v += D.escale * Ein[first + i];
          const int u0 = g0[i], u1 = g1[i];
          if (u0 >= 0) v += W0[u0];
          if (u1 >= 0) v += W1[u1];
          vec[i] = (T)v;
        }
        for (int i = hi0 + tid; i < r1; i += kSolveThreads) {
          double v = 0.0;
          const int u0 = g0[i], u1 = g1[i];
          if (u0 >= 0) v += W0[u0];
          if (u1 >= 0) v += W1[u1];
          vec[i] = (T)v;
        }
      }
      __syncthreads();
      const T* Qr = SQ + (int64_t)(n + m) * ldn;
      const int64_t woff = D.woff[s];
      for (int cb = r0; cb < r1; cb += 32) {
        const int c = cb + lane;
        T acc[K];
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] = T(0);
        if (c < r1) {
          if (c < n) col_dot<T, K>(SQ + c, ldn, 0, c + 1, vbuf, vcap, nk, acc);
          else col_dot<T, K>(Qr + (c - n), ldm, 0, n, vbuf, vcap, nk, acc);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) red[(k * kWarps + warp) * 32 + lane] = acc[k];
        __syncthreads();
        if (warp == 0 && c < r1) {
          for (int k = 0; k < nk; ++k) {
            T sum = T(0);
#pragma unroll
            for (int w2 = 0; w2 < kWarps; ++w2) sum += red[(k * kWarps + w2) * 32 + lane];
            if (c < n) D.Y[(int64_t)o[k] * D.N + first + c] = (double)sum;
            else D.W[(int64_t)o[k] * D.w_size + woff + (c - n)] = (double)(vbuf[k * vcap + c] + sum);
          }
        }
        __syncthreads();
      }
    } else if (kind == 3) {
      // transposed backward (L^T with unit diagonal): columns [r0, r1) of
      // [strict lower(SQ) ; Pb] against the own forward results and the
      // ancestors' solution
      const int32_t* ui = D.uidx + D.uoff[s];
      for (int k = 0; k < nk; ++k) {
        T* vec = vbuf + k * vcap;
        const double* Yo = D.Y + (int64_t)o[k] * D.N;
        const double* Xout = D.X + ((int64_t)o[k] * 9 + tau) * D.N;
        for (int i = r0 + tid; i < n; i += kSolveThreads) vec[i] = (T)Yo[first + i];
        for (int u = tid; u < m; u += kSolveThreads) vec[n0pad + u] = (T)Xout[ui[u]];
      }
      __syncthreads();
      const T* Pb = SQ + (int64_t)n * ldn;
      for (int cb = r0; cb < r1; cb += 32) {
        const int c = cb + lane;
        T acc[K];
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] = T(0);
        if (c < r1) {
          col_dot<T, K>(SQ + c, ldn, c + 1, n, vbuf, vcap, nk, acc);
          col_dot<T, K>(Pb + c, ldn, 0, m, vbuf + n0pad, vcap, nk, acc);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) red[(k * kWarps + warp) * 32 + lane] = acc[k];
        __syncthreads();
        if (warp == 0 && c < r1) {
          for (int k = 0; k < nk; ++k) {
            T sum = vbuf[k * vcap + c];
#pragma unroll
            for (int w2 = 0; w2 < kWarps; ++w2) sum += red[(k * kWarps + w2) * 32 + lane];
            D.X[((int64_t)o[k] * 9 + tau) * D.N + first + c] = (double)sum;
          }
        }
        __syncthreads();
      }
    } else if (kind == 0) {
      // gather each right-hand side's vector over the range the rows read
      const int lo_end = min(r1, n), hi0 = max(r0, n), w = n + m;
      const int32_t* g0 = D.ginv + D.ginv_off[s];
      const int32_t* g1 = g0 + w;
      const int c0 = D.child[2 * s], c1 = D.child[2 * s + 1];
      for (int k = 0; k < nk; ++k) {
        T* vec = vbuf + k * vcap;
        const double* Xin = D.X + ((int64_t)o[k] * 9 + tau) * D.N;
        const double* Ein = D.E ? D.E + ((int64_t)o[k] * 8 + tau) * D.N : nullptr;
        const double* Wo = D.W + (int64_t)o[k] * D.w_size;
        const double* W0 = c0 >= 0 ? Wo + D.woff[c0] : nullptr;
        const double* W1 = c1 >= 0 ? Wo + D.woff[c1] : nullptr;
        for (int i = tid; i < lo_end; i += kSolveThreads) {
          double v = Xin[first + i];
          if (Ein) v += D.escale * Ein[first + i];
          const int u0 = g0[i], u1 = g1[i];
          if (u0 >= 0) v += W0[u0];
          if (u1 >= 0) v += W1[u1];
          vec[i] = (T)v;
        }
        for (int i = hi0 + tid; i < r1; i += kSolveThreads) {
          double v = 0.0;
          const int u0 = g0[i], u1 = g1[i];
          if (u0 >= 0) v += W0[u0];
          if (u1 >= 0) v += W1[u1];
          vec[i] = (T)v;
        }
      }
      __syncthreads();
      const int64_t woff = D.woff[s];
      auto partial = [&](auto g, int i, int gl, T(&acc)[K]) {
        dot_seg_multi<T, decltype(g)::value, K>(SQ + (int64_t)i * ldn, vbuf, vcap, nk, 0, i < n ? i : n, gl, acc);
      };
      auto store = [&](int i, T(&acc)[K]) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          if (k < nk) {
            const double y = (double)(vbuf[k * vcap + i] + acc[k]);
            if (i < n) D.Y[(int64_t)o[k] * D.N + first + i] = y;
            else D.W[(int64_t)o[k] * D.w_size + woff + (i - n)] = y;
          }
      };
      const int Gl = group_lanes<T>(min(r1 - 1, n));
      ORBIT_GROUPED_ROWS_MULTI(T, K, Gl, r0, r1, warp, kWarps, partial, store);
    } else {
      const int32_t* ui = D.uidx + D.uoff[s];
      for (int k = 0; k < nk; ++k) {
        T* vec = vbuf + k * vcap;
        const double* Yo = D.Y + (int64_t)o[k] * D.N;
        const double* Xout = D.X + ((int64_t)o[k] * 9 + tau + 1) * D.N;
        for (int i = r0 + tid; i < n; i += kSolveThreads) vec[i] = (T)Yo[first + i];
        for (int u = tid; u < m; u += kSolveThreads) vec[n0pad + u] = (T)Xout[ui[u]];
      }
      __syncthreads();
      const T* Qr = SQ + (int64_t)(n + m) * ldn;
      auto partial = [&](auto g, int i, int gl, T(&acc)[K]) {
        constexpr int Gv = decltype(g)::value;
        dot_seg_multi<T, Gv, K>(SQ + (int64_t)i * ldn, vbuf, vcap, nk, i, n, gl, acc);
        dot_seg_multi<T, Gv, K>(Qr + (int64_t)i * ldm, vbuf + n0pad, vcap, nk, 0, m, gl, acc);
      };
      auto store = [&](int i, T(&acc)[K]) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          if (k < nk) D.X[((int64_t)o[k] * 9 + tau + 1) * D.N + first + i] = (double)acc[k];
      };
      const int Gl = group_lanes<T>(n - r0 + m);
      ORBIT_GROUPED_ROWS_MULTI(T, K, Gl, r0, r1, warp, kWarps, partial, store);
    }
    __syncthreads();
    if (tid == 0) {
      red_release_add(cbase + (tau * 2 + ((kind == 0 || kind == 2) ? 0 : 1)) * D.nsuper + s, 1);
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

// Bytes of each task's factor rows prefetched into L2 before its dependency
// wait at large batches: the first 48 KB (ORBIT_B200_PREFETCH_KB; 0 = the
// whole task).  With every resident CTA prefetching whole backward tasks (up
// to 64 KB at the large-batch schedule) the prefetched lines can outgrow L2
// and be fetched twice; with the evict-first row loads the 12-orbit FP32
// chain took 6.43 ms with a 48 KB window, 6.46 with 32 KB, 6.49 with 64 KB,
// 6.50 with 24 KB, 6.57 with 16 KB and 6.67 with whole tasks, while at 1 and
// 4 orbits whole tasks were fastest.
int64_t prefetch_limit_bytes() {
  static const int64_t b = [] {
    const char* e = std::getenv("ORBIT_B200_PREFETCH_KB");
    const long long kb = e ? std::atoll(e) : 48;
    return kb > 0 ? (int64_t)kb * 1024 : (int64_t)1 << 40;
  }();
  return b;
}

// Sets of task groups whose phase sequences are staggered in the claim
// order (ORBIT_B200_CHAIN_SETS, default 2; 1 = all groups in lockstep):
// measured 7.49 vs 7.62 ms for the 12-orbit FP32 chain, 12.5 vs 13.3 ms FP64,
// identical results; 3 and 4 sets were slower.
int chain_phase_sets() {
  static const int v = [] {
    const char* e = std::getenv("ORBIT_B200_CHAIN_SETS");
    const int k = e ? std::atoi(e) : 2;
    return std::max(1, std::min(k, kMaxSets));
  }();
  return v;
}

// Longest sleep between polls of a completion counter (ORBIT_B200_SPIN_NS,
// default 256 ns: 2.65 vs 2.77 ms for a single-orbit FP64 chain against a
// 1 us cap, no change at 12 orbits; 4 us was slower).
// Phases between the starts of successive staggered sets (ORBIT_B200_CHAIN_GOFF;
// unset or 0: the phases of one bin divided by the number of sets).  Any
// offset keeps every dependency claimed before its dependant (dependencies stay
// inside one orbit, hence inside one set); the last set starts at most one
// bin's phases after the first, which bounds the claim-slot table.
int chain_set_offset(int nphase, int nsets) {
  static const int v = [] {
    const char* e = std::getenv("ORBIT_B200_CHAIN_GOFF");
    return e ? std::atoi(e) : 0;
  }();
  const int g = v > 0 ? v : nphase / std::max(1, nsets);
  return std::max(1, std::min(g, nphase / std::max(1, nsets - 1)));
}

unsigned chain_spin_ns() {
  static const unsigned v = [] {
    const char* e = std::getenv("ORBIT_B200_SPIN_NS");
    const long k = e ? std::atol(e) : 256;
    return (unsigned)std::max(32L, std::min(k, 8192L));
  }();
  return v;
}

template <typename T>
int launch_chain_t(orbit_factor_s* f, double* X, int B, const int* d_orbit_ids, int trans, int tau0,
                   int tau1, const double* E, double escale, cudaStream_t st, bool never_ready = false) {
  orbit_symbolic_s* sy = f->sym;
  const Symbolic& S = sy->S;
  ChainDev<T> D;
  D.first = sy->d.first; D.n = sy->d.n; D.m = sy->d.m; D.parent = sy->d.parent;
  D.child = sy->d.child; D.uidx = sy->d.uidx; D.rel = sy->d.rel; D.ldn = sy->d.ldn; D.ldm = sy->d.ldm;
  D.ginv = sy->d.ginv; D.ginv_off = sy->d.ginv_off;
  // Right-hand sides on one factor set go through the multi-RHS kernels in
  // groups of K (row-chunk tasks, forward and transposed sweeps).
  constexpr int KM = sizeof(T) == 4 ? 4 : 2;
  const bool multi = !never_ready && f->n_sets == 1 && B >= 2 && S.max_sub_front == 0;
  const int Bt = multi ? (B + KM - 1) / KM : B;  // task groups per (node chunk, bin)
  // schedule by batch size: small chunks shorten one orbit's critical path,
  // large ones cut per-task overhead when many orbits fill the GPU
  const int ks = Bt <= 2 ? 0 : Bt <= 6 ? 1 : 2;
  const SolveSched& Q = S.sched[ks];
  const auto& q = sy->d.sched[ks];
  D.nch_f = trans ? q.nchunk_fwdT : q.nchunk_fwd;
  D.nch_b = trans ? q.nchunk_bwdT : q.nchunk_bwd;
  D.level = sy->d.level;
  D.sub_front = S.max_sub_front;
  D.uoff = sy->d.uoff; D.fac_off = sy->d.fac_off; D.woff = sy->d.woff;
  D.items = trans ? q.sitems + Q.items_per_bin : q.sitems;
  D.phase_off = trans ? q.phase_offT : q.phase_off;
  D.nphase = 2 * S.nlevels;
  if (D.nphase > kMaxPhases) {
    set_last_error("chained solve: supernode tree deeper than the kernel's phase table");
    return ORBIT_ERR_INTERNAL;
  }
  D.items_per_bin = trans ? Q.items_per_binT : Q.items_per_bin;
  D.nsuper = S.nsuper;
  D.N = S.N; D.fac_size = S.fac_size; D.w_size = S.w_size;
  D.factors = reinterpret_cast<const T*>(f->factors);
  D.X = X; D.E = E; D.escale = escale; D.Y = f->Ybuf; D.W = f->Wbuf;
  D.counters = f->counters; D.task_counter = f->task_counter; D.status = f->status;
  D.orbit_ids = d_orbit_ids; D.B = Bt; D.Borb = B; D.tau0 = tau0; D.tau1 = tau1; D.trans = trans;
  D.set_of = f->set_of; D.n_bins = f->n_bins;
  D.total = (tau1 - tau0) * D.items_per_bin * Bt;
  D.spin_limit = never_ready ? 20000LL : 4000000LL;  // bounded: a few seconds of sleeps (<= 1 us each)
  D.never_ready = never_ready ? 1 : 0;
  D.prefetch = (sizeof(T) == 4 || B <= 6) ? 1 : 0;
  // the window bounds the prefetch only where the prefetched lines of all
  // resident CTAs outgrow L2 (large batches); small batches prefetch whole tasks
  D.prefetch_bytes = Bt > 6 ? prefetch_limit_bytes() : ((int64_t)1 << 40);
  // evict-first factor loads only where no two solve slots share a factor set
  D.stream_ef = 1;
  {
    std::vector<char> seen((size_t)std::max(f->n_sets, 1), 0);
    for (int o = 0; o < f->n_orbits && D.stream_ef; ++o) {
      const int st_o = f->h_set_of[o];
      if (st_o < 0 || st_o >= f->n_sets || seen[st_o]) D.stream_ef = 0;
      else seen[st_o] = 1;
    }
  }
  D.spin_ns = chain_spin_ns();
  D.ngroups = std::max(1, std::min(Bt, chain_phase_sets()));
  D.goff = D.ngroups > 1 ? chain_set_offset(D.nphase, D.ngroups) : 0;
  if (D.total <= 0) return ORBIT_OK;
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->counters, 0, sizeof(int) * (size_t)f->n_orbits * 16 * S.nsuper, st));
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->task_counter, 0, sizeof(int), st));
  const size_t smem =
      sizeof(T) * ((size_t)kWarps * 32 + std::max<size_t>(S.max_front + 8, (size_t)kWarps * ((S.max_sub_front + 7) & ~3)) + 8);
  const bool sub = S.max_sub_front > 0;
  const void* kfn = trans ? (sub ? (const void*)k_chain<T, true, true> : (const void*)k_chain<T, true, false>)
                          : (sub ? (const void*)k_chain<T, false, true> : (const void*)k_chain<T, false, false>);
  {
    int r0 = allow_max_smem(kfn);
    if (r0) return r0;
  }
  int dev = 0, sms = 0, occ = 0;
  ORBIT_CUDA_TRY(cudaGetDevice(&dev));
  ORBIT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (multi) {
    const int vcap = (S.max_front + 8 + 3) & ~3;
    const size_t msmem = sizeof(T) * ((size_t)KM * vcap + (size_t)KM * kWarps * 32);
    {
      int r0 = allow_max_smem((const void*)k_chain_multi<T, KM>);
      if (r0) return r0;
    }
    ORBIT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_chain_multi<T, KM>, kSolveThreads, msmem));
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
    k_chain_multi<T, KM><<<grid, kSolveThreads, msmem, st>>>(D, vcap);
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
  ORBIT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kSolveThreads, smem));
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
  if (trans) {
    if (sub) k_chain<T, true, true><<<grid, kSolveThreads, smem, st>>>(D);
    else k_chain<T, true, false><<<grid, kSolveThreads, smem, st>>>(D);
  } else {
    if (sub) k_chain<T, false, true><<<grid, kSolveThreads, smem, st>>>(D);
    else k_chain<T, false, false><<<grid, kSolveThreads, smem, st>>>(D);
  }
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

// One chain launch whose first task waits for a completion count that is
// never reached: exercises the bounded wait, the status word and the orderly
// exit of every CTA.
int chain_wait_selftest(orbit_factor_s* f, const int* d_orbit_ids, cudaStream_t st) {
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->status, 0, sizeof(int), st));
  int rc = f->precision == ORBIT_PREC_FP32
               ? launch_chain_t<float>(f, f->X, 1, d_orbit_ids, 0, 0, f->n_bins, nullptr, 0.0, st, true)
               : launch_chain_t<double>(f, f->X, 1, d_orbit_ids, 0, 0, f->n_bins, nullptr, 0.0, st, true);
  if (rc) return rc;
  ORBIT_CUDA_TRY(cudaMemcpyAsync(f->h_status, f->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  ORBIT_CUDA_TRY(cudaStreamSynchronize(st));
  const int code = *f->h_status;
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->status, 0, sizeof(int), st));
  ORBIT_CUDA_TRY(cudaStreamSynchronize(st));
  return code;
}

}  // namespace orbit
