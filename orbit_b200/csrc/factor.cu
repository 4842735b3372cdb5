// K3: batched numeric factorization of A = I + dtau (T + diag(sink)) on the
// dense supernodes of the symbolic analysis.
//
// Replaces the reference's per-bin sparse LU (_factor_one_bin ->
// umfpack_di_numeric / scipy splu; orbit/core/orbit.py:79-96,
// orbit/core/solve.py:210-243).  A is strictly row-diagonally dominant
// (I plus an M-matrix times dtau), so no pivoting is needed; the reference's
// SuperLU runs also pivot on the diagonal (perm_r == perm_c).
//
// Each supernode front F = [F11 F12; F21 F22] (own rows first, then the
// ancestor rows of its update set) is assembled from the stencil and the
// children's Schur complements (extend-add), partially factored by a blocked
// right-looking LU, and stored for the solve as
//   SQ = strict_lower(inv(L11)) + upper(inv(U11))   (n x n)
//   Pb = -L21 inv(L11)                              (m x n)
//   Qr = -inv(U11) U12                              (n x m)
// so that every supernode step of the triangular solves is a dense
// matrix-vector product with no intra-supernode dependency.  The Schur
// complement F22 - L21 U12 stays in the front for the parent.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <type_traits>

#include "common.cuh"
#include "handles.h"
#include "tc.cuh"

namespace orbit {

namespace {

constexpr int kThreads = 256;
constexpr int kLdS = 68;  // shared-memory tile stride (16-byte aligned rows)

template <typename T>
struct Ld {
  const T* p;
  int ld, rows, cols, mask, tri;
  __device__ __forceinline__ T operator()(int r, int c) const {
    if (r >= rows || c >= cols) return T(0);
    if (mask == 1) {
      int d = c - r;
      if (d > tri) return T(0);
      if (d == tri) return T(1);
    } else if (mask == 2) {
      if (c - r < tri) return T(0);
    }
    return p[(int64_t)r * ld + c];
  }
};

// 4 consecutive elements from 16-byte aligned shared memory.
template <typename T>
__device__ __forceinline__ void lds4(const T* p, T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}

template <typename T>
struct LdS {  // operand held in shared memory (ld kLdS)
  const T* p;
  int rows, cols;
  __device__ __forceinline__ T operator()(int r, int c) const {
    if (r >= rows || c >= cols) return T(0);
    return p[r * kLdS + c];
  }
};

// acc (64 x 64; thread (ty, tx) holds rows 4 ty + i, columns 4 tx + j) +=
// A (64 x K) B (K x 64) in 16-deep slabs
// staged through shared memory; the next slab's operands are loaded into
// registers while the current slab is multiplied.
template <typename T, class LA, class LB>
__device__ __forceinline__ void mma_tile(T (&acc)[4][4], int K, const LA& la, const LB& lb, T* As,
                                         T* Bs) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * kThreads;
      ra[q] = la(e >> 4, k0 + (e & 15));
      rb[q] = lb(k0 + (e >> 6), e & 63);
    }
  };
  if (K > 0) fetch(0);
  for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * kThreads;
      As[(e & 15) * kLdS + (e >> 4)] = ra[q];
      Bs[(e >> 6) * kLdS + (e & 63)] = rb[q];
    }
    __syncthreads();
    if (k0 + 16 < K) fetch(k0 + 16);
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      T a[4], b[4];
      lds4(As + kk * kLdS + 4 * ty, a);
      lds4(Bs + kk * kLdS + 4 * tx, b);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
}

template <typename T>
__device__ __forceinline__ void zero_acc(T (&acc)[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
}

struct FactorDev {
  const int32_t *n, *m, *parent, *child, *rel, *ldn, *ldm, *ldf;
  const int32_t* ginv;
  const int64_t* ginv_off;
  const int64_t *uoff, *fac_off, *front_off;
  const int4* items;
  int64_t fac_size, front_buf;
  int group;  // instances per front group
  const int64_t* tc_pack_off;
  int64_t tc_pack_stride;  // floats per instance
  int tc_min_n;            // nodes with n >= tc_min_n and m > 0 take the tensor-core pipeline
};

// True for the supernodes whose factorization the tensor-core pipeline
// completes: their pivot LU stays inside F11 and the triangle copies and
// CUDA-core panel products skip them.
__device__ __forceinline__ bool tc_node(const FactorDev& D, int n, int m) { return m > 0 && n >= D.tc_min_n; }


template <typename T>
__global__ void k_scatter(T* fronts, int64_t stride, const int64_t* ent_pos, const int32_t* ent_src,
                          int64_t e0, int64_t ne, const double* const* Tp, const double* const* Dp,
                          int inst_base, int64_t N, double dtau) {
  const int inst = inst_base + blockIdx.y;
  const double* Tv = Tp[inst];
  const double* Dv = Dp[inst];
  T* f = fronts + (int64_t)blockIdx.y * stride;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    int32_t src = ent_src[e0 + e];
    int d = (int)(src / N);
    int64_t cell = src - (int64_t)d * N;
    double t = Tv[src];
    double val = d == 0 ? 1.0 + dtau * (t + (Dv ? Dv[cell] : 0.0)) : dtau * t;
    f[ent_pos[e0 + e]] += (T)val;
  }
}

// FP64 copy of the assembled stencil of A for iterative refinement.
__global__ void k_copy_A(double* A, const double* const* Tp, const double* const* Dp,
                         int inst_base, int64_t N, double dtau) {
  const int inst = inst_base + blockIdx.y;
  const double* Tv = Tp[inst];
  const double* Dv = Dp[inst];
  double* out = A + (int64_t)inst * 7 * N;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 7 * N;
       e += (int64_t)gridDim.x * blockDim.x) {
    double t = Tv[e];
    out[e] = e < N ? 1.0 + dtau * (t + (Dv ? Dv[e] : 0.0)) : dtau * t;
  }
}

// Front assembly by gather: row i of the front of s is the sum of the two
// children's Schur-complement rows mapped through the inverse extend-add maps
// (zero where no child contributes), written once together with its padding
// columns.  The stencil entries are added afterwards (k_scatter).  One warp
// per row, four consecutive columns per lane: the maps are read from shared
// memory as int4, the row is stored with 16-byte stores (rows start 16-byte
// aligned), and the children's rows are read in increasing column order.
template <typename T>
__global__ void __launch_bounds__(256) k_assemble(FactorDev D, T* fr, const T* fr_child, int64_t i0) {
  extern __shared__ int4 sinv4[];  // map of child 0 at [0, wp), child 1 at [wp, 2 wp)
  int32_t* sinv = reinterpret_cast<int32_t*>(sinv4);
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, r0 = it.y, r1 = it.z;
  const int n = D.n[s], m = D.m[s], w = n + m, ldf = D.ldf[s];
  const int wp = (w + 3) & ~3;  // <= ldf
  const int32_t* gi = D.ginv + D.ginv_off[s];
  for (int j = threadIdx.x; j < 2 * wp; j += blockDim.x) {
    const int q = j >= wp, jj = j - q * wp;
    sinv[j] = jj < w ? gi[q * w + jj] : -1;
  }
  __syncthreads();
  T* F = fr + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  const T* Sc[2] = {nullptr, nullptr};
  int ldc[2] = {0, 0};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int c = D.child[2 * s + q];
    if (c >= 0) {
      ldc[q] = D.ldf[c];
      Sc[q] = fr_child + (int64_t)blockIdx.y * D.front_buf + D.front_off[c] + (int64_t)D.n[c] * ldc[q] + D.n[c];
    }
  }
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  constexpr int VW = 16 / sizeof(T);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = r0 + warp; i < r1; i += blockDim.x / 32) {
    const int u0 = sinv[i], u1 = sinv[wp + i];
    const T* s0 = u0 >= 0 ? Sc[0] + (int64_t)u0 * ldc[0] : nullptr;
    const T* s1 = u1 >= 0 ? Sc[1] + (int64_t)u1 * ldc[1] : nullptr;
    T* row = F + (int64_t)i * ldf;
    // two 128-column chunks per iteration: all gathers in flight before the stores
    for (int jb = 4 * lane; jb < ldf; jb += 256) {
      T v[2][4];
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        const int j0 = jb + 128 * g;
#pragma unroll
        for (int h = 0; h < 4; ++h) v[g][h] = T(0);
        if (j0 < wp) {
          if (s0) {
            const int4 c = sinv4[j0 >> 2];
            if (c.x >= 0) v[g][0] += s0[c.x];
            if (c.y >= 0) v[g][1] += s0[c.y];
            if (c.z >= 0) v[g][2] += s0[c.z];
            if (c.w >= 0) v[g][3] += s0[c.w];
          }
          if (s1) {
            const int4 c = sinv4[(wp + j0) >> 2];
            if (c.x >= 0) v[g][0] += s1[c.x];
            if (c.y >= 0) v[g][1] += s1[c.y];
            if (c.z >= 0) v[g][2] += s1[c.z];
            if (c.w >= 0) v[g][3] += s1[c.w];
          }
        }
      }
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        const int j0 = jb + 128 * g;
        if (j0 >= ldf) break;
#pragma unroll
        for (int h = 0; h < 4; h += VW) {
          V x;
          if constexpr (VW == 4) {
            x.x = v[g][0]; x.y = v[g][1]; x.z = v[g][2]; x.w = v[g][3];
          } else {
            x.x = v[g][h]; x.y = v[g][h + 1];
          }
          *reinterpret_cast<V*>(row + j0 + h) = x;
        }
      }
    }
  }
}

template <typename T>
__global__ void k_panel(FactorDev D, T* fronts, const T* factors, int64_t i0, int p0,
                        int inst_base) {
  extern __shared__ unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);
  T* Bs = As + 16 * kLdS;
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, kind = it.y, ch = it.z;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s], ldn = D.ldn[s];
  const int nb = min(64, n - p0);
  const int q0 = p0 + nb;
  const int lim = tc_node(D, n, m) ? n : n + m;  // last row / column the panels reach
  if (q0 + 64 * ch >= lim) return;
  T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  const T* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s];
  T acc[4][4];
  zero_acc(acc);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  if (kind == 0) {
    const int c0 = q0 + 64 * ch, w = min(64, lim - c0);
    Ld<T> A{SQ + (int64_t)p0 * ldn + p0, ldn, nb, nb, 1, 0};
    Ld<T> B{F + (int64_t)p0 * ldf + c0, ldf, nb, w, 0, 0};
    mma_tile(acc, nb, A, B, As, Bs);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int r = 4 * ty + i, c = 4 * tx + j;
        if (r < nb && c < w) F[(int64_t)(p0 + r) * ldf + c0 + c] = acc[i][j];
      }
  } else {
    const int r0 = q0 + 64 * ch, h = min(64, lim - r0);
    Ld<T> A{F + (int64_t)r0 * ldf + p0, ldf, h, nb, 0, 0};
    Ld<T> B{SQ + (int64_t)p0 * ldn + p0, ldn, nb, nb, 2, 0};
    mma_tile(acc, nb, A, B, As, Bs);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int r = 4 * ty + i, c = 4 * tx + j;
        if (r < h && c < nb) F[(int64_t)(r0 + r) * ldf + p0 + c] = acc[i][j];
      }
  }
}

// Register-tiled GEMM of one output tile: C (h x w) -= A (h x K) B (K x w), or
// C = -A B when `assign`; outputs with r >= skip_r and c >= skip_c are left
// untouched.  Each of 256 threads owns a TM x TN block of outputs;
// the A and B slabs (128 x 16 and 16 x BN) go through shared memory with
// 16-byte reads of the outer-product operands, and the next slab is prefetched
// into registers while the current one is multiplied.
template <typename T, int TM, int TN, int BN>
__device__ __forceinline__ void gemm_tile(const T* __restrict__ A, int lda, const T* __restrict__ B,
                                          int ldb, T* C, int ldc, int K, int h, int w, bool assign,
                                          T* As, T* Bs, int skip_r = 1 << 30, int skip_c = 1 << 30) {
  constexpr int BM = 128, BK = 16;
  constexpr int LDA = BM + 4, LDB = BN + 4;
  constexpr int AL = BM * BK / 256, BL = BK * BN / 256;
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  constexpr int VW = 16 / sizeof(T);
  const int tid = threadIdx.x, tx = tid % (BN / TN), ty = tid / (BN / TN);
  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
  T ra[AL], rb[BL];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < AL; ++q) {
      const int e = tid + q * 256, r = e / BK, kk = e % BK;
      ra[q] = (r < h && k0 + kk < K) ? A[(int64_t)r * lda + k0 + kk] : T(0);
    }
#pragma unroll
    for (int q = 0; q < BL; ++q) {
      const int e = tid + q * 256, kk = e / BN, c = e % BN;
      rb[q] = (c < w && k0 + kk < K) ? B[(int64_t)(k0 + kk) * ldb + c] : T(0);
    }
  };
  load(0);
  for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
    for (int q = 0; q < AL; ++q) {
      const int e = tid + q * 256;
      As[(e % BK) * LDA + e / BK] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < BL; ++q) {
      const int e = tid + q * 256;
      Bs[(e / BN) * LDB + e % BN] = rb[q];
    }
    __syncthreads();
    if (k0 + BK < K) load(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < TM; i += VW) {
        const V t = *reinterpret_cast<const V*>(As + kk * LDA + ty * TM + i);
        if constexpr (sizeof(T) == 4) {
          a[i] = t.x; a[i + 1] = t.y; a[i + 2] = t.z; a[i + 3] = t.w;
        } else {
          a[i] = t.x; a[i + 1] = t.y;
        }
      }
#pragma unroll
      for (int j = 0; j < TN; j += VW) {
        const V t = *reinterpret_cast<const V*>(Bs + kk * LDB + tx * TN + j);
        if constexpr (sizeof(T) == 4) {
          b[j] = t.x; b[j + 1] = t.y; b[j + 2] = t.z; b[j + 3] = t.w;
        } else {
          b[j] = t.x; b[j + 1] = t.y;
        }
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int r = ty * TM + i;
    if (r >= h) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int c = tx * TN + j;
      if (c < w && !(r >= skip_r && c >= skip_c)) {
        if (assign) C[(int64_t)r * ldc + c] = -acc[i][j];
        else C[(int64_t)r * ldc + c] -= acc[i][j];
      }
    }
  }
}

// C tile (128 x 128) -= / = - A B with K in [k0, K): FP32 as one 128x128
// register tile, FP64 as two 128x64 halves.
template <typename T>
__device__ __forceinline__ void gemm_128(const T* A, int lda, const T* B, int ldb, T* C, int ldc, int K,
                                         int h, int w, bool assign, T* smem, int skip_r = 1 << 30,
                                         int skip_c = 1 << 30) {
  T* As = smem;
  T* Bs = smem + 16 * (128 + 4);
  if constexpr (sizeof(T) == 4) {
    gemm_tile<T, 8, 8, 128>(A, lda, B, ldb, C, ldc, K, h, w, assign, As, Bs, skip_r, skip_c);
  } else {
    for (int half = 0; half < 2; ++half) {
      const int cc = 64 * half;
      if (cc >= w) break;
      gemm_tile<T, 8, 4, 64>(A, lda, B + cc, ldb, C + cc, ldc, K, h, min(64, w - cc), assign, As, Bs, skip_r,
                             skip_c - cc);
    }
  }
}

// Trailing update after pivot block [p0, q0): the 128 x 128 tile (tr, tc) of
// the rows and columns beyond q0 gets -= L[:, p0:q0] U[p0:q0, :], except its
// part inside F22 (rows and columns >= n), which the Schur pass updates once.
template <typename T>
__global__ void __launch_bounds__(256, 2) k_update2(FactorDev D, T* fronts, int64_t i0, int p0) {
  extern __shared__ unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, tr = it.y, tc = it.z;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s];
  const int nb = min(64, n - p0);
  const int q0 = p0 + nb;
  const int r0 = q0 + 128 * tr, c0 = q0 + 128 * tc;
  const int lim = tc_node(D, n, m) ? n : n + m;
  if (r0 >= lim || c0 >= lim) return;
  T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  gemm_128<T>(F + (int64_t)r0 * ldf + p0, ldf, F + (int64_t)p0 * ldf + c0, ldf, F + (int64_t)r0 * ldf + c0, ldf,
              nb, min(128, lim - r0), min(128, lim - c0), false, sm, n - r0, n - c0);
}

// Schur complement of a front: F22 -= L21 U12 (K = n), one 128 x 128 tile per CTA.
template <typename T>
__global__ void __launch_bounds__(256, 2) k_schur(FactorDev D, T* fronts, int64_t i0) {
  extern __shared__ unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, tr = it.y, tc = it.z;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s];
  T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  const int r0 = 128 * tr, c0 = 128 * tc;
  gemm_128<T>(F + (int64_t)(n + r0) * ldf, ldf, F + n + c0, ldf, F + (int64_t)(n + r0) * ldf + n + c0, ldf, n,
              min(128, m - r0), min(128, m - c0), false, sm);
}

// Dense copy of one triangle of the explicit inverses into the (no longer
// needed) pivot block of the front: kind 0 -> unit-lower inv(L11), kind 1 ->
// upper inv(U11), zeros elsewhere, so the panel products are plain GEMMs.
template <typename T>
__global__ void k_tri_copy(FactorDev D, T* fronts, const T* factors, int64_t i0, int kind, int inst_base) {
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, rb = it.y;
  const int n = D.n[s], ldf = D.ldf[s], ldn = D.ldn[s];
  if (tc_node(D, n, D.m[s])) return;
  T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  const T* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s];
  for (int r = rb * 16 + (threadIdx.x >> 5); r < min(n, rb * 16 + 16); r += 8)
    for (int c = threadIdx.x & 31; c < n; c += 32) {
      T v;
      if (kind == 0) v = c < r ? SQ[(int64_t)r * ldn + c] : (c == r ? T(1) : T(0));
      else v = c >= r ? SQ[(int64_t)r * ldn + c] : T(0);
      F[(int64_t)r * ldf + c] = v;
    }
}

// Panel products with the dense triangles in F11:
// kind 0: Pb (m x n) = -L21 inv(L11), tile (tr of m, tc of n), K from 128 tc;
// kind 1: Qr (n x m) = -inv(U11) U12, tile (tr of n, tc of m), K from 128 tr.
template <typename T>
__global__ void __launch_bounds__(256, 2) k_prod2(FactorDev D, const T* fronts, T* factors, int64_t i0, int kind,
                                               int inst_base) {
  extern __shared__ unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, tr = it.y, tc = it.z;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s], ldn = D.ldn[s], ldm = D.ldm[s];
  if (tc_node(D, n, m)) return;
  const T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  T* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s];
  const int r0 = 128 * tr, c0 = 128 * tc;
  if (kind == 0) {
    T* Pb = SQ + (int64_t)n * ldn;
    gemm_128<T>(F + (int64_t)(n + r0) * ldf + c0, ldf, F + (int64_t)c0 * ldf + c0, ldf, Pb + (int64_t)r0 * ldn + c0,
                ldn, n - c0, min(128, m - r0), min(128, n - c0), true, sm);
  } else {
    T* Qr = SQ + (int64_t)(n + m) * ldn;
    gemm_128<T>(F + (int64_t)r0 * ldf + r0, ldf, F + (int64_t)r0 * ldf + n + c0, ldf, Qr + (int64_t)r0 * ldm + c0,
                ldm, n - r0, min(128, n - r0), min(128, m - c0), true, sm);
  }
}

template <typename T>
__global__ void k_inv(FactorDev D, const T* fronts, T* factors, int64_t i0, int inst_base) {
  extern __shared__ unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);
  T* Bs = As + 16 * kLdS;
  T* Xs = Bs + 16 * kLdS;
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, kind = it.y, jb = it.z, t = it.w;
  const int n = D.n[s], ldf = D.ldf[s], ldn = D.ldn[s];
  const T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  T* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
  zero_acc(acc);
  if (kind == 0) {
    // Linv block (t, jb): -Linv_tt * sum_{k=jb}^{t-1} L_tk Linv_k,jb, the sum as
    // one product over the contiguous columns 64 jb .. 64 t of L and rows of
    // Linv (the unit-lower mask only bites in the first, diagonal block)
    const int r0 = 64 * t, h = min(64, n - r0), c0 = 64 * jb, K = 64 * (t - jb);
    {
      Ld<T> A{F + (int64_t)r0 * ldf + c0, ldf, h, K, 0, 0};
      Ld<T> B{SQ + (int64_t)c0 * ldn + c0, ldn, K, 64, 1, 0};
      mma_tile(acc, K, A, B, As, Bs);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) Xs[(4 * ty + i) * kLdS + 4 * tx + j] = acc[i][j];
    __syncthreads();
    zero_acc(acc);
    Ld<T> A{SQ + (int64_t)r0 * ldn + r0, ldn, h, h, 1, 0};
    LdS<T> B{Xs, h, 64};
    mma_tile(acc, h, A, B, As, Bs);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int r = 4 * ty + i, c = 4 * tx + j;
        if (r < h) SQ[(int64_t)(r0 + r) * ldn + c0 + c] = -acc[i][j];
      }
  } else {
    // Uinv block (jb, t): -(sum_{k=jb}^{t-1} Uinv_jb,k U_kt) Uinv_tt, the sum as
    // one product (the upper mask only bites in the first, diagonal block)
    const int r0 = 64 * jb, c0 = 64 * t, w = min(64, n - c0), K = 64 * (t - jb);
    {
      Ld<T> A{SQ + (int64_t)r0 * ldn + r0, ldn, 64, K, 2, 0};
      Ld<T> B{F + (int64_t)r0 * ldf + c0, ldf, K, w, 0, 0};
      mma_tile(acc, K, A, B, As, Bs);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) Xs[(4 * ty + i) * kLdS + 4 * tx + j] = acc[i][j];
    __syncthreads();
    zero_acc(acc);
    LdS<T> A{Xs, 64, w};
    Ld<T> B{SQ + (int64_t)c0 * ldn + c0, ldn, w, w, 2, 0};
    mma_tile(acc, w, A, B, As, Bs);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int r = 4 * ty + i, c = 4 * tx + j;
        if (c < w) SQ[(int64_t)(r0 + r) * ldn + c0 + c] = -acc[i][j];
      }
  }
}

// ---- one-CTA fronts ----
//
// A supernode with n <= 64 pivots whose pivot-block inverses and panels fit
// in shared memory is factored whole by one CTA, which does what the DIAG,
// PANEL, UPDATE, INV, TRIL/TRIU, PRODL/PRODU and SCHUR launches do for the
// larger ones: unpivoted LU of F11 with the explicit inverses (stored as SQ),
// X = inv(U11) inv(L11) (= inv(F11)), Pb = -F21 X, Qr = -X F12 and
// F22 += Pb F12 (the products the tensor-core pipeline forms).  The deepest
// levels of the dissection are thousands of such fronts per instance, which
// the multi-launch path runs at a few per cent of the GPU.  Shared memory
// (ldq = round_up(n, 4) + 4, ldl = round_up(m, 4); front_smem_elems):
//   Q  [n][ldq]  strict lower inv(L11), upper inv(U11) (= SQ), then X
//   Qt [n][ldq]  the staged F11 until the inverses are formed, then Q^T, then X^T
//   Lt [n][ldl]  F21^T, then Pb^T
//   U  [n][ldl]  F12
//   ex [2][4][64] exchange slots of the pivot steps

// Asynchronous copy of one element from global to shared memory.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(sizeof(T)) : "memory");
}

template <typename T>
__device__ __forceinline__ void sts4(T* p, T a, T b, T c, T d) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
  } else {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
    *reinterpret_cast<double2*>(p + 2) = make_double2(c, d);
  }
}

// One step k of a 4 x 4 block product: acc(i, q) += A(r + i, k) B(k, c + q)
// with A read as At[k * lda + r] and B as Bm[k * ldb + c]; with MASK the
// terms outside k >= r + i (A = inv(U11)) and k > c + q (B = inv(L11)) vanish.
template <typename T, bool MASK>
__device__ __forceinline__ void fb_step(const T* At, int lda, const T* Bm, int ldb, int k, int r, int c,
                                        T (&acc)[4][4]) {
  T a[4], b[4];
  lds4(At + k * lda + r, a);
  lds4(Bm + k * ldb + c, b);
  if (MASK) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (!(k >= r + i)) a[i] = T(0);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (!(k > c + q)) b[q] = T(0);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[i][q] = fma(a[i], b[q], acc[i][q]);
}

// Dense 4 x 4 block product over k < K (block at (r, c), multiples of 4).
template <typename T>
__device__ __forceinline__ void front_block(const T* At, int lda, const T* Bm, int ldb, int K, int r, int c,
                                            T (&acc)[4][4]) {
  zero_acc(acc);
#pragma unroll 4
  for (int k = 0; k < K; ++k) fb_step<T, false>(At, lda, Bm, ldb, k, r, c, acc);
}

// X(r + i, c + q) = sum over k >= max(r + i, c + q) of inv(U11)(r + i, k)
// inv(L11)(k, c + q): the unit diagonal of inv(L11) gives the k = c + q term
// inv(U11)(r + i, c + q), the rest runs over k > c with both triangles masked
// only next to the block's diagonals.  inv(U11)(r, k) = Q[r][k] = Qt[k][r]
// (k >= r), inv(L11)(k, c) = Q[k][c] (k > c).
template <typename T>
__device__ __forceinline__ void front_x_block(const T* Q, const T* Qt, int ldq, int n, int r, int c,
                                              T (&acc)[4][4]) {
  zero_acc(acc);
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (c + q < n) {
      T v[4];
      lds4(Qt + (c + q) * ldq + r, v);
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i][q] = (c + q >= r + i) ? v[i] : T(0);
    }
  const int k0 = max(r, c + 1), k1 = min(n, max(r + 3, c + 4));
  for (int k = k0; k < k1; ++k) fb_step<T, true>(Qt, ldq, Q, ldq, k, r, c, acc);
#pragma unroll 4
  for (int k = max(k0, k1); k < n; ++k) fb_step<T, false>(Qt, ldq, Q, ldq, k, r, c, acc);
}

// Unpivoted LU of the staged F11 (Dm) with inv(L11) and inv(U11)^T formed in
// the same pivot steps, one barrier per step; the result goes to Q (strict
// lower inv(L11), upper inv(U11)) and Qt = Q^T.  Thread (ty, tx) holds rows
// ty + 16a and columns tx + 16b (a, b < G, n <= 16 G) of A (F11, becoming
// the LU), X (inv(L11)) and Z (inv(U11)^T, by forward substitution on U^T:
// row k of U is final at step k).  At step k the holders of row k publish
// its A, X and Z values, those of column k its A values; after the barrier
// every thread applies, for its rows i > k,
//   A(i, j) -= l_i A(k, j)  (j > k; l_i = A(i, k) / A(k, k) is stored at j = k)
//   X(i, j) -= l_i X(k, j)
//   Z(i, j) -= A(k, i) z_j  (z_j = Z(k, j) / A(k, k), stored in row k).
// Row and column groups of 16 that a step cannot touch are skipped; the
// exchange slots alternate between two sets so that one barrier per step
// orders every write after the previous step's reads.
template <typename T, int G>
__device__ __forceinline__ void front_lu(const T* Dm, T* Q, T* Qt, T* ex, int n, int ldq, int* status,
                                         T* LUo = nullptr) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T A[G][G], X[G][G], Z[G][G];
#pragma unroll
  for (int a = 0; a < G; ++a)
#pragma unroll
    for (int b = 0; b < G; ++b) {
      const int i = ty + 16 * a, j = tx + 16 * b;
      A[a][b] = (i < n && j < n) ? Dm[i * ldq + j] : T(0);
      X[a][b] = Z[a][b] = (i == j) ? T(1) : T(0);
    }
  for (int k = 0; k < n; ++k) {
    T* pr = ex + (k & 1) * 256;
    T* lc = pr + 64;
    T* xr = lc + 64;
    T* zr = xr + 64;
    const int kr = k & 15, kg = k >> 4;
    if (ty == kr) {
#pragma unroll
      for (int a = 0; a < G; ++a)
        if (a == kg) {
#pragma unroll
          for (int b = 0; b < G; ++b) {
            const int j = tx + 16 * b;
            pr[j] = A[a][b];
            xr[j] = X[a][b];
            zr[j] = Z[a][b];
          }
        }
    }
    if (tx == kr) {
#pragma unroll
      for (int b = 0; b < G; ++b)
        if (b == kg) {
#pragma unroll
          for (int a = 0; a < G; ++a) lc[ty + 16 * a] = A[a][b];
        }
    }
    __syncthreads();
    const T piv = pr[k];
    if (tid == 0 && (!(piv == piv) || piv == T(0) || isinf((double)piv))) raise_status(status, ORBIT_ERR_PIVOT);
    const T rp = T(1) / piv;
    T pj[G], xj[G], zj[G];
#pragma unroll
    for (int b = 0; b < G; ++b) {
      const int j = tx + 16 * b;
      pj[b] = j > k ? pr[j] : T(0);
      xj[b] = xr[j];
      zj[b] = zr[j] * rp;
    }
#pragma unroll
    for (int a = 0; a < G; ++a) {
      if (16 * a + 15 < k) continue;  // every row of the group is above the pivot
      const int i = ty + 16 * a;
      const bool below = i > k;
      const T l = below ? lc[i] * rp : T(0);
      const T u = below ? pr[i] : T(0);
#pragma unroll
      for (int b = 0; b < G; ++b) {
        if (16 * b + 15 > k) A[a][b] -= l * pj[b];  // columns j > k exist in the group
        if (16 * b <= k) {                          // X(k, j), Z(k, j) vanish for j > k
          X[a][b] -= l * xj[b];
          Z[a][b] = (i == k) ? zj[b] : Z[a][b] - u * zj[b];
        }
      }
      if (below && tx == kr) {
#pragma unroll
        for (int b = 0; b < G; ++b)
          if (b == kg) A[a][b] = l;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < G; ++a)
#pragma unroll
    for (int b = 0; b < G; ++b) {
      const int i = ty + 16 * a, j = tx + 16 * b;
      if (i < n && j < n) {
        if (i > j) {
          Q[i * ldq + j] = X[a][b];
          Qt[j * ldq + i] = X[a][b];
        }
        if (i >= j) {
          Q[j * ldq + i] = Z[a][b];
          Qt[i * ldq + j] = Z[a][b];
        }
        if (LUo) LUo[i * ldq + j] = A[a][b];
      }
    }
}

// Diagonal block (p0 .. p0 + nb) of a blocked supernode: its LU back into the
// front and strict_lower(inv(L)) + upper(inv(U)) into SQ, by the one-pass
// register LU of the one-CTA fronts.
template <typename T>
__global__ void __launch_bounds__(256) k_diag(FactorDev D, T* fronts, T* factors, int64_t i0, int p0, int inst_base,
                                              int* status) {
  extern __shared__ unsigned char smem_raw[];
  constexpr int ldq = kNB + 4;
  T* Dm = reinterpret_cast<T*>(smem_raw);
  T* Q = Dm + kNB * ldq;
  T* Qt = Q + kNB * ldq;
  T* ex = Qt + kNB * ldq;
  const int s = D.items[i0 + blockIdx.x].x;
  const int n = D.n[s];
  const int nb = min(kNB, n - p0);
  const int ldf = D.ldf[s], ldn = D.ldn[s];
  T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s] + (int64_t)p0 * ldf + p0;
  T* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s] + (int64_t)p0 * ldn + p0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int r = warp; r < nb; r += kThreads / 32)
    for (int c = lane; c < nb; c += 32) cp_async_elem(Dm + r * ldq + c, F + (int64_t)r * ldf + c);
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  if (nb <= 16) front_lu<T, 1>(Dm, Q, Qt, ex, nb, ldq, status, Dm);
  else if (nb <= 32) front_lu<T, 2>(Dm, Q, Qt, ex, nb, ldq, status, Dm);
  else if (nb <= 48) front_lu<T, 3>(Dm, Q, Qt, ex, nb, ldq, status, Dm);
  else front_lu<T, 4>(Dm, Q, Qt, ex, nb, ldq, status, Dm);
  __syncthreads();
  for (int r = warp; r < nb; r += kThreads / 32)
    for (int c = lane; c < nb; c += 32) {
      F[(int64_t)r * ldf + c] = Dm[r * ldq + c];
      SQ[(int64_t)r * ldn + c] = Q[r * ldq + c];
    }
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 2 : 3) k_front(FactorDev D, T* fronts, T* factors, int64_t i0, int inst_base,
                                               int* status) {
  extern __shared__ unsigned char smem_raw[];
  const int s = D.items[i0 + blockIdx.x].x;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s], ldn = D.ldn[s], ldm = D.ldm[s];
  const int ldq = ((n + 3) & ~3) + 4, ldl = (m + 3) & ~3;
  T* Q = reinterpret_cast<T*>(smem_raw);
  T* Qt = Q + n * ldq;
  T* Lt = Qt + n * ldq;
  T* U = Lt + n * ldl;
  T* ex = U + n * ldl;
  T* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  T* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s];
  T* Pb = SQ + (int64_t)n * ldn;
  T* Qr = SQ + (int64_t)(n + m) * ldn;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // 1. F11 (into Qt's space), F12 and F21^T into shared memory by
  // asynchronous element copies (rows by warps, columns by lanes), all in
  // flight before the wait
  for (int r = warp; r < n; r += kThreads / 32) {
    const T* row = F + (int64_t)r * ldf;
    for (int c = lane; c < n + m; c += 32) cp_async_elem(c < n ? Qt + r * ldq + c : U + r * ldl + (c - n), row + c);
  }
  for (int r = warp; r < m; r += kThreads / 32) {
    const T* row = F + (int64_t)(n + r) * ldf;
    for (int c = lane; c < n; c += 32) cp_async_elem(Lt + c * ldl + r, row + c);
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();

  // 2. LU and both triangular inverses into Q / Qt, register blocks sized to n
  if (n <= 16) front_lu<T, 1>(Qt, Q, Qt, ex, n, ldq, status);
  else if (n <= 32) front_lu<T, 2>(Qt, Q, Qt, ex, n, ldq, status);
  else if (n <= 48) front_lu<T, 3>(Qt, Q, Qt, ex, n, ldq, status);
  else front_lu<T, 4>(Qt, Q, Qt, ex, n, ldq, status);
  __syncthreads();

  // 3. SQ to the factor storage; X = inv(U11) inv(L11) into registers, then
  // over Q (and X^T over Qt) once every thread has read them
  for (int r = warp; r < n; r += kThreads / 32)
    for (int c = lane; c < n; c += 32) SQ[(int64_t)r * ldn + c] = Q[r * ldq + c];
  const int wn = (n + 3) >> 2;        // threads across n (4 columns each)
  const int wo = kThreads / wn;       // threads across m
  const int an = tid % wn, ao = tid / wn;
  {
    const bool act = tid < wn * wn;
    const int r = 4 * (tid / wn), c = 4 * (tid % wn);
    T x[4][4];
    if (act) front_x_block<T>(Q, Qt, ldq, n, r, c, x);
    __syncthreads();
    if (act)
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (r + i < n && c + q < n) {
            Q[(r + i) * ldq + c + q] = x[i][q];
            Qt[(c + q) * ldq + r + i] = x[i][q];
          }
  }
  __syncthreads();

  // 4. Pb = -F21 X to the factor storage (padding columns untouched) and,
  // in place of F21^T, as Pb^T for the Schur complement; a block of Pb rows
  // reads only its own columns of Lt, so one barrier before its stores suffices
  for (int rb = 0; rb < m; rb += 4 * wo) {
    const int r = rb + 4 * ao, c = 4 * an;
    const bool act = ao < wo && r < m;
    T acc[4][4];
    if (act) front_block<T>(Lt, ldl, Q, ldq, n, r, c, acc);
    __syncthreads();
    if (act) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (c + q < n) sts4(Lt + (c + q) * ldl + r, -acc[0][q], -acc[1][q], -acc[2][q], -acc[3][q]);
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (r + i < m) {
          T* o = Pb + (int64_t)(r + i) * ldn + c;
          if (c + 3 < n) {
            sts4(o, -acc[i][0], -acc[i][1], -acc[i][2], -acc[i][3]);
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (c + q < n) o[q] = -acc[i][q];
          }
        }
    }
  }
  __syncthreads();

  // 5. Qr = -X F12 to the factor storage, then F22 += Pb F12 in the front
  for (int cb = 0; cb < m; cb += 4 * wo) {
    const int r = 4 * an, c = cb + 4 * ao;
    if (ao < wo && c < m) {
      T acc[4][4];
      front_block<T>(Qt, ldq, U, ldl, n, r, c, acc);
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (r + i < n) {
          T* o = Qr + (int64_t)(r + i) * ldm + c;
          if (c + 3 < m) {
            sts4(o, -acc[i][0], -acc[i][1], -acc[i][2], -acc[i][3]);
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (c + q < m) o[q] = -acc[i][q];
          }
        }
    }
  }
  {
    // 64 x 64 tiles of F22; the next tile's current values are loaded while
    // this tile's products run
    const int tx = tid & 15, ty = tid >> 4;
    const int mt = (m + 63) / 64;
    T* F22 = F + (int64_t)n * ldf + n;
    auto load_tile = [&](int t, T (&v)[4][4]) {
      const int r = (t / mt) * 64 + 4 * ty, c = (t % mt) * 64 + 4 * tx;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          v[i][q] = (r + i < m && c + q < m) ? F22[(int64_t)(r + i) * ldf + c + q] : T(0);
    };
    T cv[4][4], cn[4][4];
    load_tile(0, cv);
    for (int t = 0; t < mt * mt; ++t) {
      if (t + 1 < mt * mt) load_tile(t + 1, cn);
      const int r = (t / mt) * 64 + 4 * ty, c = (t % mt) * 64 + 4 * tx;
      if (r < m && c < m) {
        T acc[4][4];
        front_block<T>(Lt, ldl, U, ldl, n, r, c, acc);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (r + i < m && c + q < m) F22[(int64_t)(r + i) * ldf + c + q] = cv[i][q] + acc[i][q];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) cv[i][q] = cn[i][q];
    }
  }
}

// ---- tensor-core pipeline (fp32 factors) ----
//
// For the large supernodes the pivot LU stays inside F11, the inverses
// inv(L11), inv(U11) are formed as for every node, and then
//   X  = inv(U11) inv(L11)      (= inv(F11))
//   Pb = -F21 X                 (= -L21 inv(L11))
//   Qr = -X F12                 (= -inv(U11) U12)
//   F22 += Pb F12               (= F22 - L21 U12)
// run on the 5th-generation tensor cores with split tf32 operands
// (x = hi + lo, hi = tf32(x), lo = tf32(x - hi); products accumulated as
// hi*hi + hi*lo + lo*hi in fp32 in tensor memory), which keeps the error of an
// fp32 GEMM.  k_tc_pack writes each operand tile once, already split and in the
// swizzled shared-memory layout; the GEMM moves whole 16 KB hi/lo tile pairs
// with single bulk copies.

static_assert(tc::kCols == kTcK && tc::kTileFloats == kTcTileFloats, "packed tile geometry");

// Float offset of tile (t, kb) of a node's pack region (tiles of 2 x 2048
// floats, hi then lo): 0 F21 (mt x kt), 1 F12^T (mt x kt), 2 inv(U11)
// (nt x kt), 3 inv(L11)^T (nt x kt), 4 X (nt x kt), 5 X^T (nt x kt), 6 Pb
// (mt x kt).  Regions 0-3 are written by k_tc_pack, 4-6 by GEMM epilogues.
__device__ __forceinline__ int64_t tc_tile(int region, int t, int kb, int mt, int nt, int kt) {
  const int64_t M = (int64_t)mt * kt, Nn = (int64_t)nt * kt;
  const int64_t base = region == 0   ? 0
                       : region == 1 ? M
                       : region == 2 ? 2 * M
                       : region == 3 ? 2 * M + Nn
                       : region == 4 ? 2 * M + 2 * Nn
                       : region == 5 ? 2 * M + 3 * Nn
                                     : 2 * M + 4 * Nn;
  return (base + (int64_t)t * kt + kb) * (2 * tc::kTileFloats);
}

// Split four values into tf32 hi/lo and store them as one 16-byte chunk of
// the hi plane and of the lo plane.
__device__ __forceinline__ void store_split4(float* tile, int off, float a, float b, float c, float d) {
  float4 hi, lo;
  hi.x = tc::to_tf32(a); lo.x = tc::to_tf32(a - hi.x);
  hi.y = tc::to_tf32(b); lo.y = tc::to_tf32(b - hi.y);
  hi.z = tc::to_tf32(c); lo.z = tc::to_tf32(c - hi.z);
  hi.w = tc::to_tf32(d); lo.w = tc::to_tf32(d - hi.w);
  *reinterpret_cast<float4*>(tile + off) = hi;
  *reinterpret_cast<float4*>(tile + tc::kTileFloats + off) = lo;
}

// A run of kTcPackRun 128 x 16 operand tiles of one row tile: op 0 F21 and
// op 2 inv(U11) (A side: rows x K, read along rows), op 1 F12^T and op 3
// inv(L11)^T with its unit diagonal (B side: columns x K, read down columns).
// Every load of the run is issued before the first store.
__global__ void __launch_bounds__(256) k_tc_pack(FactorDev D, const float* fronts, const float* factors,
                                                 float* pack, int64_t i0, int inst_base) {
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, op = it.y, t = it.z, kb0 = it.w;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s], ldn = D.ldn[s];
  const int mt = (m + 127) / 128, nt = (n + 127) / 128, kt = (n + tc::kCols - 1) / tc::kCols;
  const float* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  const float* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s];
  const int region = op;
  const int rows = op <= 1 ? m : n;
  const bool bside = op == 1 || op == 3;
  float* dst0 = pack + (int64_t)blockIdx.y * D.tc_pack_stride + D.tc_pack_off[s];
  constexpr int kPer = tc::kRows * (tc::kCols / 4) / 256;  // 16-byte chunks per thread and tile
  float v[kTcPackRun][kPer][4];
#pragma unroll
  for (int h = 0; h < kTcPackRun; ++h)
#pragma unroll
    for (int p = 0; p < kPer; ++p) {
      // A side: 4 consecutive threads read one 64-byte row segment; B side:
      // consecutive threads read consecutive columns of one source row.
      const int q = threadIdx.x + 256 * p;
      const int r = bside ? q & 127 : q >> 2;
      const int c = bside ? q >> 7 : q & 3;
      const int row = t * tc::kRows + r;
      const int k = (kb0 + h) * tc::kCols + c * 4;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int kk = k + u;
        float x = 0.f;
        if (row < rows && kk < n) {
          switch (op) {
            case 0: x = F[(int64_t)(n + row) * ldf + kk]; break;
            case 1: x = F[(int64_t)kk * ldf + n + row]; break;
            case 2: x = kk >= row ? SQ[(int64_t)row * ldn + kk] : 0.f; break;
            default: x = row < kk ? SQ[(int64_t)kk * ldn + row] : (row == kk ? 1.f : 0.f); break;
          }
        }
        v[h][p][u] = x;
      }
    }
#pragma unroll
  for (int h = 0; h < kTcPackRun; ++h) {
    if (kb0 + h >= kt) break;
    float* dst = dst0 + tc_tile(region, t, kb0 + h, mt, nt, kt);
#pragma unroll
    for (int p = 0; p < kPer; ++p) {
      const int q = threadIdx.x + 256 * p;
      const int r = bside ? q & 127 : q >> 2;
      const int c = bside ? q >> 7 : q & 3;
      store_split4(dst, tc::swz(r, c * 4), v[h][p][0], v[h][p][1], v[h][p][2], v[h][p][3]);
    }
  }
}

constexpr int kTcStages = 2;
constexpr int kTcStageBytes = 4 * tc::kTileBytes;  // A hi, A lo, B hi, B lo
constexpr size_t kTcSmem = (size_t)kTcStages * kTcStageBytes + 512;
constexpr long long kTcWaitLimit = 1LL << 22;

// One 128 x 128 output tile per CTA of job 0 (X, written only as the X and
// X^T operand packs), 1 (Pb, into the factor storage and as the Pb operand
// pack), 2 (Qr, into the factor storage) or 3 (F22 += Pb F12).  Three CTAs per SM (64 KB ring and 128 TMEM columns each) so that one
// CTA's epilogue overlaps the others' main loops (measured faster than two
// CTAs with 3-stage rings).  Warp 0 lane 0 streams the k-blocks into a
// 2-stage ring, warp 1 lane 0 issues the MMAs, all four warps
// read the accumulator back (warp w owns TMEM lanes 32w..32w+31 = tile rows)
// and stage it through shared memory so that the output goes row by row,
// coalesced.  Every wait is bounded; on a timeout the CTA lets its copies
// land, skips the update, raises ORBIT_ERR_TIMEOUT and frees its tensor memory.
__global__ void __launch_bounds__(128, 3) k_gemm_tc(FactorDev D, float* fronts, float* factors, float* pack,
                                                    int64_t i0, int inst_base, int* status) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t full[kTcStages], empty[kTcStages], done;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const uint32_t raw = tc::smem_u32(smem_raw);
  unsigned char* sbuf = smem_raw + ((512u - (raw & 511u)) & 511u);
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, tr = it.y, tcol = it.z, job = it.w;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s], ldn = D.ldn[s], ldm = D.ldm[s];
  const int mt = (m + 127) / 128, nt = (n + 127) / 128, kt = (n + tc::kCols - 1) / tc::kCols;
  const int ra = job == 0 ? 2 : job == 1 ? 0 : job == 2 ? 4 : 6;
  const int rb = job == 0 ? 3 : job == 1 ? 5 : 1;
  const int M = (job == 0 || job == 2) ? n : m;
  const int N = (job == 0 || job == 1) ? n : m;
  // X = inv(U11) inv(L11): both factors vanish below k = max(row, column)
  const int kb0 = job == 0 ? (tc::kRows / tc::kCols) * max(tr, tcol) : 0;
  const int nk = kt - kb0;
  float* pk2 = pack + (int64_t)blockIdx.y * D.tc_pack_stride + D.tc_pack_off[s];
  const float* pk = pk2;
  const float* pa = pk + tc_tile(ra, tr, kb0, mt, nt, kt);
  const float* pb = pk + tc_tile(rb, tcol, kb0, mt, nt, kt);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kTcStages; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    tc::mbar_init(&done, 1);
    failed = 0;
    tc::fence_barrier_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(&tmem_base, 128);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  if (threadIdx.x == 0) {
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int st = kb % kTcStages;
      if (kb >= kTcStages && !tc::mbar_wait(&empty[st], ((kb / kTcStages) - 1) & 1, kTcWaitLimit)) {
        failed = 1;
        break;
      }
      unsigned char* sb = sbuf + st * kTcStageBytes;
      tc::mbar_arrive_expect_tx(&full[st], kTcStageBytes);
      tc::bulk_g2s(sb, pa + (int64_t)kb * (2 * tc::kTileFloats), 2 * tc::kTileBytes, &full[st]);
      tc::bulk_g2s(sb + 2 * tc::kTileBytes, pb + (int64_t)kb * (2 * tc::kTileFloats), 2 * tc::kTileBytes,
                   &full[st]);
      issued = kb + 1;
    }
    // every issued copy has landed before this CTA may finish
    for (int kb = max(0, issued - kTcStages); kb < issued; ++kb)
      if (!tc::mbar_wait(&full[kb % kTcStages], (kb / kTcStages) & 1, kTcWaitLimit)) failed = 1;
  } else if (job == 3 && warp >= 2) {
    // the F22 tile this CTA updates does not depend on the GEMM: warps 2-3
    // ask L2 for it while the main loop runs (one 128-byte line per request)
    const int rows = min(128, M - tr * tc::kRows), cols = min(128, N - tcol * 128);
    const float* C0 = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s] +
                      (int64_t)(n + tr * tc::kRows) * ldf + n + tcol * 128;
    for (int q = threadIdx.x - 64; q < rows * 5; q += 64) {
      const int r = q / 5, seg = q - r * 5;
      const float* a = C0 + (int64_t)r * ldf + min(seg * 32, cols - 1);  // stays inside the row
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
    }
  } else if (threadIdx.x == 32) {
    const uint32_t idesc = tc::idesc_tf32(128, 128);
    for (int kb = 0; kb < nk; ++kb) {
      const int st = kb % kTcStages;
      if (!tc::mbar_wait(&full[st], (kb / kTcStages) & 1, kTcWaitLimit)) {
        failed = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t a = tc::smem_u32(sbuf + st * kTcStageBytes);
      const uint32_t ahi = a, alo = a + tc::kTileBytes, bhi = a + 2 * tc::kTileBytes, blo = a + 3 * tc::kTileBytes;
#pragma unroll
      for (int kk = 0; kk < tc::kCols / 8; ++kk) {
        const uint32_t o = kk * 32;  // 8 tf32 along K inside the 64-byte swizzled row
        tc::mma_tf32(tmem, tc::sw64_desc(ahi + o), tc::sw64_desc(bhi + o), idesc, (kb | kk) != 0);
        tc::mma_tf32(tmem, tc::sw64_desc(ahi + o), tc::sw64_desc(blo + o), idesc, 1);
        tc::mma_tf32(tmem, tc::sw64_desc(alo + o), tc::sw64_desc(bhi + o), idesc, 1);
      }
      tc::mma_commit(&empty[st]);
    }
    tc::mma_commit(&done);
  }
  const bool ok = tc::mbar_wait(&done, 0, kTcWaitLimit);
  tc::fence_after_sync();
  const int good = __syncthreads_and(ok ? 1 : 0) && !failed;
  if (good) {
    float* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
    float* SQ = factors + (int64_t)(inst_base + blockIdx.y) * D.fac_size + D.fac_off[s];
    float* C = nullptr;
    int ldc = 0;
    if (job == 0) {
    } else if (job == 1) {
      C = SQ + (int64_t)n * ldn;
      ldc = ldn;
    } else if (job == 2) {
      C = SQ + (int64_t)(n + m) * ldn;
      ldc = ldm;
    } else {
      C = F + (int64_t)n * ldf + n;
      ldc = ldf;
    }
    // the ring is idle now: each warp transposes its 32 x 32 accumulator
    // blocks through a private padded buffer
    float* sw = reinterpret_cast<float*>(sbuf) + warp * 32 * 33;
    const int rows = min(32, M - tr * tc::kRows - warp * 32);
    const int cols = job == 0 ? 0 : min(128, N - tcol * 128);
    // operand packs written here cover the K extent of the next GEMMs
    // (zero-padded rows and columns included: the accumulator is zero there)
    const int kcols = job <= 1 ? min(128, tc::kCols * kt - 128 * tcol) : 0;
    if (C) C += (int64_t)(tr * tc::kRows + warp * 32) * ldc + tcol * 128;
    for (int cc = 0; cc < 4 && cc * 32 < max(cols, kcols); ++cc) {
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc * 32), v);
      if (job <= 1) {
        // A-side pack of this row block: X (job 0) or Pb = -acc (job 1)
        const float sg = job == 0 ? 1.f : -1.f;
        const int rl = warp * 32 + lane;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int kb = tcol * (tc::kRows / tc::kCols) + cc * 2 + h;
          if (kb < kt) {
            float* tile = pk2 + tc_tile(job == 0 ? 4 : 6, tr, kb, mt, nt, kt);
#pragma unroll
            for (int q = 0; q < 4; ++q)
              store_split4(tile, tc::swz(rl, q * 4), sg * v[h * 16 + q * 4], sg * v[h * 16 + q * 4 + 1],
                           sg * v[h * 16 + q * 4 + 2], sg * v[h * 16 + q * 4 + 3]);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) sw[lane * 33 + j] = v[j];
      __syncwarp();
      if (job == 0) {
        // B-side pack X^T: pack row = X column, K = X row
        const int crow = cc * 32 + lane;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int kb = tr * (tc::kRows / tc::kCols) + warp * 2 + h;
          if (kb < kt) {
            float* tile = pk2 + tc_tile(5, tcol, kb, mt, nt, kt);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int r = h * 16 + q * 4;
              store_split4(tile, tc::swz(crow, q * 4), sw[r * 33 + lane], sw[(r + 1) * 33 + lane],
                           sw[(r + 2) * 33 + lane], sw[(r + 3) * 33 + lane]);
            }
          }
        }
      }
      const int col = cc * 32 + lane;
      if (col < cols) {
        if (job == 3) {
          // all 32 rows' loads in flight before any update
          float c[32];
#pragma unroll
          for (int u = 0; u < 32; ++u)
            if (u < rows) c[u] = C[(int64_t)u * ldc + col];
#pragma unroll
          for (int u = 0; u < 32; ++u)
            if (u < rows) C[(int64_t)u * ldc + col] = c[u] + sw[u * 33 + lane];
        } else {
          const float sg = job == 0 ? 1.f : -1.f;
          for (int r = 0; r < rows; ++r) C[(int64_t)r * ldc + col] = sg * sw[r * 33 + lane];
        }
      }
      __syncwarp();
    }
  } else if (threadIdx.x == 0) {
    raise_status(status, ORBIT_ERR_TIMEOUT);
  }
  // On a timeout, MMAs already issued may still write this CTA's tensor
  // memory: wait once more (bounded) for their commit before the columns are
  // released.  The status word then carries ORBIT_ERR_TIMEOUT and the handle's
  // factors are not to be used.
  if (!ok) tc::mbar_wait(&done, 0, kTcWaitLimit);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(tmem, 128);
}

// Trailing update of the blocked pivot LU on the tensor cores (fp32 fronts):
// the 128 x 128 tile (tr, tc) beyond the pivot block [p0, q0) gets
// C -= L[:, p0:q0] U[p0:q0, :] (K = nb <= 64) with split tf32 operands, the
// part inside F22 (rows and columns >= n) left to the Schur pass, as k_update2
// does on the CUDA cores.  All 128 threads load their operand rows (A: one
// tile row each, 16-byte loads along K; B: one tile column each, coalesced
// across the warp), split them into tf32 hi/lo and store them in the 64-byte
// swizzled layout the MMA descriptors read; two k-blocks of 16 per round,
// then one thread issues the MMAs into the tensor-memory accumulator.  Three
// CTAs per SM overlap one tile's loads and epilogue with the others' MMAs.
// Every wait is bounded; on a timeout the CTA leaves the tile untouched,
// raises ORBIT_ERR_TIMEOUT and frees its tensor memory.
constexpr int kUpdKb = 2;                                        // k-blocks of 16 per round
constexpr size_t kUpdSmem = (size_t)kUpdKb * kTcStageBytes + 512;

__global__ void __launch_bounds__(128, 3) k_update_tc(FactorDev D, float* fronts, int64_t i0, int p0,
                                                      int* status) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t full, done;
  __shared__ uint32_t tmem_base;
  const uint32_t raw = tc::smem_u32(smem_raw);
  unsigned char* sbuf = smem_raw + ((512u - (raw & 511u)) & 511u);
  const int4 it = D.items[i0 + blockIdx.x];
  const int s = it.x, tr = it.y, tcl = it.z;
  const int n = D.n[s], m = D.m[s], ldf = D.ldf[s];
  const int nb = min(64, n - p0);
  const int q0 = p0 + nb;
  const int r0 = q0 + 128 * tr, c0 = q0 + 128 * tcl;
  const int lim = tc_node(D, n, m) ? n : n + m;
  if (r0 >= lim || c0 >= lim) return;  // uniform over the CTA
  const int M = min(128, lim - r0), N = min(128, lim - c0);
  float* F = fronts + (int64_t)blockIdx.y * D.front_buf + D.front_off[s];
  const float* A = F + (int64_t)r0 * ldf + p0;  // M x nb, row-major
  const float* B = F + (int64_t)p0 * ldf + c0;  // nb x N, row-major
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, t = threadIdx.x;
  if (t == 0) {
    tc::mbar_init(&full, 128);
    tc::mbar_init(&done, 1);
    tc::fence_barrier_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(&tmem_base, 128);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_tf32(128, 128);
  const int nkb = (nb + tc::kCols - 1) / tc::kCols;
  bool ok = true;
  uint32_t ph = 0;
  for (int kb0 = 0; kb0 < nkb && ok; kb0 += kUpdKb) {
    const int nr = min(kUpdKb, nkb - kb0);
    for (int h = 0; h < nr; ++h) {
      float* At = reinterpret_cast<float*>(sbuf + h * kTcStageBytes);
      float* Bt = At + 2 * tc::kTileFloats;
      const int k0 = (kb0 + h) * tc::kCols;
      // A row t: 16 values along K, 16-byte loads (rows start 16-byte aligned
      // and p0, k0 are multiples of 16; a load that starts below nb stays inside
      // the padded row); entries at k >= nb belong to the next pivot columns
      // and are zeroed
      float a[16];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (t < M && k0 + 4 * q < nb) v = *reinterpret_cast<const float4*>(A + (int64_t)t * ldf + k0 + 4 * q);
        const int kq = k0 + 4 * q;
        a[4 * q] = kq < nb ? v.x : 0.f;
        a[4 * q + 1] = kq + 1 < nb ? v.y : 0.f;
        a[4 * q + 2] = kq + 2 < nb ? v.z : 0.f;
        a[4 * q + 3] = kq + 3 < nb ? v.w : 0.f;
      }
      // B column t: 16 values down K (consecutive t read consecutive columns)
      float b[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) b[k] = (t < N && k0 + k < nb) ? B[(int64_t)(k0 + k) * ldf + t] : 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        store_split4(At, tc::swz(t, 4 * q), a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
        store_split4(Bt, tc::swz(t, 4 * q), b[4 * q], b[4 * q + 1], b[4 * q + 2], b[4 * q + 3]);
      }
    }
    tc::fence_proxy_async();
    tc::mbar_arrive(&full);
    if (t == 32) {
      if (tc::mbar_wait(&full, ph, kTcWaitLimit)) {
        tc::fence_after_sync();
        for (int h = 0; h < nr; ++h) {
          const uint32_t a0 = tc::smem_u32(sbuf + h * kTcStageBytes);
          const uint32_t ahi = a0, alo = a0 + tc::kTileBytes, bhi = a0 + 2 * tc::kTileBytes,
                         blo = a0 + 3 * tc::kTileBytes;
#pragma unroll
          for (int kk = 0; kk < tc::kCols / 8; ++kk) {
            const uint32_t o = kk * 32;
            tc::mma_tf32(tmem, tc::sw64_desc(ahi + o), tc::sw64_desc(bhi + o), idesc, ((kb0 + h) | kk) != 0);
            tc::mma_tf32(tmem, tc::sw64_desc(ahi + o), tc::sw64_desc(blo + o), idesc, 1);
            tc::mma_tf32(tmem, tc::sw64_desc(alo + o), tc::sw64_desc(bhi + o), idesc, 1);
          }
        }
      }
      tc::mma_commit(&done);
    }
    // the round's MMAs have read the operands before the buffers are refilled
    if (!tc::mbar_wait(&done, ph, kTcWaitLimit)) ok = false;
    ph ^= 1u;
    tc::fence_after_sync();
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
  }
  if (ok) {
    // each warp stages its 32 x 32 accumulator blocks through shared memory
    // so that the update goes row by row, coalesced
    float* sw = reinterpret_cast<float*>(sbuf) + warp * 32 * 33;
    const int rows = min(32, M - warp * 32);
    for (int cc = 0; cc < 4 && cc * 32 < N; ++cc) {
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc * 32), v);
#pragma unroll
      for (int j = 0; j < 32; ++j) sw[lane * 33 + j] = v[j];
      __syncwarp();
      const int col = cc * 32 + lane;
      if (col < N) {
        float* C = F + (int64_t)(r0 + warp * 32) * ldf + c0 + col;
        const bool f22_col = c0 + col >= n;
        float c[32];
#pragma unroll
        for (int u = 0; u < 32; ++u)
          if (u < rows) c[u] = C[(int64_t)u * ldf];
#pragma unroll
        for (int u = 0; u < 32; ++u)
          if (u < rows && !(f22_col && r0 + warp * 32 + u >= n)) C[(int64_t)u * ldf] = c[u] - sw[u * 33 + lane];
      }
      __syncwarp();
    }
  } else if (t == 0) {
    raise_status(status, ORBIT_ERR_TIMEOUT);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(tmem, 128);
}

inline int clamp_grid(int64_t blocks) {
  if (blocks < 1) return 1;
  if (blocks > (1 << 20)) return 1 << 20;
  return (int)blocks;
}

template <typename T>
int run_factor_t(orbit_factor_s* f, int n_active, double dtau, cudaStream_t st) {
  orbit_symbolic_s* sy = f->sym;
  const Symbolic& S = sy->S;
  FactorDev D;
  D.n = sy->d.n; D.m = sy->d.m; D.parent = sy->d.parent; D.child = sy->d.child; D.rel = sy->d.rel;
  D.ginv = sy->d.ginv; D.ginv_off = sy->d.ginv_off;
  D.ldn = sy->d.ldn; D.ldm = sy->d.ldm; D.ldf = sy->d.ldf;
  D.uoff = sy->d.uoff; D.fac_off = sy->d.fac_off; D.front_off = sy->d.front_off;
  D.items = sy->d.fitems;
  D.fac_size = S.fac_size;
  D.front_buf = S.front_buf_size;
  D.group = f->front_group;
  D.tc_pack_off = sy->d.tc_pack_off;
  D.tc_pack_stride = S.tc_pack_size;
  D.tc_min_n = INT_MAX;
  T* factors = reinterpret_cast<T*>(f->factors);
  T* fronts = reinterpret_cast<T*>(f->fronts);
  const int n_inst = n_active * f->n_bins;
  const size_t sm_gemm = 2 * 16 * kLdS * sizeof(T);
  const size_t sm_inv = sm_gemm + 64 * kLdS * sizeof(T);
  const size_t sm_diag = (3 * kNB * (kNB + 4) + 512) * sizeof(T);
  const size_t sm_schur = 16 * (128 + 4) * sizeof(T) + 16 * (128 + 4) * sizeof(T);
  { int _r = allow_max_smem((const void*)k_schur<T>); if (_r) return _r; }
  bool use_tc = false, tc_update = false;
  if constexpr (std::is_same<T, float>::value) {
    const char* e = std::getenv("ORBIT_B200_TC");
    use_tc = f->tc_pack != nullptr && !(e && e[0] == '0');
    if (use_tc) {
      int _r = allow_max_smem((const void*)k_gemm_tc);
      if (_r) return _r;
      D.tc_min_n = S.tc_min_n;
      // trailing updates of the blocked pivot LU on the tensor cores as well,
      // unless ORBIT_B200_TC_UPDATE=0
      const char* eu = std::getenv("ORBIT_B200_TC_UPDATE");
      tc_update = !(eu && eu[0] == '0');
      if (tc_update) {
        _r = allow_max_smem((const void*)k_update_tc);
        if (_r) return _r;
      }
    }
  }
  { int _r = allow_max_smem((const void*)k_prod2<T>); if (_r) return _r; }
  { int _r = allow_max_smem((const void*)k_update2<T>); if (_r) return _r; }
  { int _r = allow_max_smem((const void*)k_diag<T>); if (_r) return _r; }
  { int _r = allow_max_smem((const void*)k_inv<T>); if (_r) return _r; }
  { int _r = allow_max_smem((const void*)k_front<T>); if (_r) return _r; }
  {
    dim3 g(clamp_grid((7 * S.N + 255) / 256), n_inst);
    k_copy_A<<<g, 256, 0, st>>>(f->A_stencil, f->d_Tptr, f->d_Dptr, 0, S.N, dtau);
    note_launch();
    ORBIT_CUDA_TRY(cudaGetLastError());
  }
  for (int base = 0; base < n_inst; base += f->front_group) {
    const int G = std::min(f->front_group, n_inst - base);
    for (const FactorLaunch& L : S.fsched) {
      T* cur = fronts + (int64_t)(L.level & 1) * f->front_group * S.front_buf_size;
      T* chl = fronts + (int64_t)((L.level + 1) & 1) * f->front_group * S.front_buf_size;
      if (L.items <= 0) continue;
      switch (L.kind) {
        case FactorLaunch::ASSEMBLE: {
          dim3 g((unsigned)L.items, G);
          k_assemble<T><<<g, 256, sizeof(int32_t) * 2 * (S.max_front + 4), st>>>(D, cur, chl, L.item_off);
          note_launch();
          break;
        }
        case FactorLaunch::SCATTER: {
          dim3 g(clamp_grid((L.items + 255) / 256), G);
          k_scatter<T><<<g, 256, 0, st>>>(cur, S.front_buf_size, sy->d.ent_pos, sy->d.ent_src,
                                          L.item_off, L.items, f->d_Tptr, f->d_Dptr, base, S.N, dtau);
          note_launch();
          break;
        }
        case FactorLaunch::FRONT: {
          dim3 g((unsigned)L.items, G);
          k_front<T><<<g, kThreads, (size_t)L.p0 * sizeof(T), st>>>(D, cur, factors, L.item_off, base, f->status);
          note_launch();
          break;
        }
        case FactorLaunch::DIAG: {
          dim3 g((unsigned)L.items, G);
          k_diag<T><<<g, kThreads, sm_diag, st>>>(D, cur, factors, L.item_off, L.p0, base, f->status);
          note_launch();
          break;
        }
        case FactorLaunch::PANEL: {
          dim3 g((unsigned)L.items, G);
          k_panel<T><<<g, kThreads, sm_gemm, st>>>(D, cur, factors, L.item_off, L.p0, base);
          note_launch();
          break;
        }
        case FactorLaunch::UPDATE: {
          dim3 g((unsigned)L.items, G);
          bool done_tc = false;
          if constexpr (std::is_same<T, float>::value) {
            if (use_tc && tc_update) {
              k_update_tc<<<g, 128, kUpdSmem, st>>>(D, cur, L.item_off, L.p0, f->status);
              done_tc = true;
            }
          }
          if (!done_tc) k_update2<T><<<g, 256, sm_schur, st>>>(D, cur, L.item_off, L.p0);
          note_launch();
          break;
        }
        case FactorLaunch::TC_PACK: {
          if constexpr (std::is_same<T, float>::value) {
            if (use_tc) {
              dim3 g((unsigned)L.items, G);
              k_tc_pack<<<g, 256, 0, st>>>(D, cur, factors, f->tc_pack, L.item_off, base);
              note_launch();
            }
          }
          break;
        }
        case FactorLaunch::TC_GEMM: {
          if constexpr (std::is_same<T, float>::value) {
            if (use_tc) {
              dim3 g((unsigned)L.items, G);
              k_gemm_tc<<<g, 128, kTcSmem, st>>>(D, cur, factors, f->tc_pack, L.item_off, base, f->status);
              note_launch();
            }
          }
          break;
        }
        case FactorLaunch::SCHUR: {
          const int64_t n_cc = use_tc ? L.p0 : L.items;
          if (n_cc > 0) {
            dim3 g((unsigned)n_cc, G);
            k_schur<T><<<g, 256, sm_schur, st>>>(D, cur, L.item_off);
            note_launch();
          }
          break;
        }
        case FactorLaunch::INV: {
          dim3 g((unsigned)L.items, G);
          k_inv<T><<<g, kThreads, sm_inv, st>>>(D, cur, factors, L.item_off, base);
          note_launch();
          break;
        }
        case FactorLaunch::TRIL:
        case FactorLaunch::TRIU: {
          dim3 g((unsigned)L.items, G);
          k_tri_copy<T><<<g, 256, 0, st>>>(D, cur, factors, L.item_off, L.kind == FactorLaunch::TRIL ? 0 : 1, base);
          note_launch();
          break;
        }
        case FactorLaunch::PRODL:
        case FactorLaunch::PRODU: {
          dim3 g((unsigned)L.items, G);
          k_prod2<T><<<g, 256, sm_schur, st>>>(D, cur, factors, L.item_off, L.kind == FactorLaunch::PRODL ? 0 : 1, base);
          note_launch();
          break;
        }
        default:
          break;
      }
      ORBIT_CUDA_TRY(cudaGetLastError());
    }
  }
  return ORBIT_OK;
}

}  // namespace

int run_factor(orbit_factor_s* f, int n_active, double dtau, cudaStream_t st) {
  if (f->precision == ORBIT_PREC_FP32) return run_factor_t<float>(f, n_active, dtau, st);
  return run_factor_t<double>(f, n_active, dtau, st);
}

}  // namespace orbit
