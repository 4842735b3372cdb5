// The outer closure loop around the orbit solve: the 7-D ISORROPIA lookup
// table query and the vector work of the Anderson step.
//
// LUT query (IsorropiaLUT.query, orbit/core/isorropia_lut.py:116-147): the
// reference evaluates scipy's RegularGridInterpolator, method "linear",
// fill_value None, on float32 tables over seven ascending axes (total SO4,
// total NH, total NO3, crustal Ca, sea-salt Na, T, RH).  Here one thread per
// query point locates its cell on every axis by binary search (clamped to the
// first and last interval, so points outside the table extrapolate linearly
// from the edge cell, as fill_value None does), forms the 2^7 corner weights
// and accumulates the float32 table values in double precision; the outputs
// are clipped as the reference clips them (fractions to [0, 1], water >= 0).
//
// Anderson step (AndersonAccelerator, orbit/core/closure_iteration.py:
// 568-694): the state vectors stay on the device; the step needs the dot
// products of a few difference vectors (the m x m least-squares system) and a
// linear combination of them, both provided here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace orbit {
namespace {

constexpr int kLutDims = 7;
constexpr int kMaxVecs = 16;

struct LutArgs {
  const double* axis[kLutDims];
  int n[kLutDims];
  int64_t stride[kLutDims];
  const float* field[4];
};

__device__ __forceinline__ int find_cell(const double* a, int n, double x) {
  // largest i in [0, n - 2] with a[i] <= x (0 below the axis, n - 2 above)
  int lo = 0, hi = n - 2;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void k_lut_query(LutArgs A, int64_t npts, const double* __restrict__ pts, double* __restrict__ out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  int idx[kLutDims];
  double t[kLutDims];
  bool nan_in = false;
  for (int d = 0; d < kLutDims; ++d) {
    const double x = pts[(int64_t)d * npts + p];
    nan_in |= !(x == x);
    const int i = find_cell(A.axis[d], A.n[d], x);
    const double a0 = A.axis[d][i], a1 = A.axis[d][i + 1];
    idx[d] = i;
    t[d] = (x - a0) / (a1 - a0);
  }
  for (int f = 0; f < 4; ++f) {
    double v = NAN;
    if (A.field[f] && !nan_in) {
      v = 0.0;
      for (int corner = 0; corner < (1 << kLutDims); ++corner) {
        double w = 1.0;
        int64_t off = 0;
#pragma unroll
        for (int d = 0; d < kLutDims; ++d) {
          const int b = (corner >> (kLutDims - 1 - d)) & 1;
          w *= b ? t[d] : 1.0 - t[d];
          off += (int64_t)(idx[d] + b) * A.stride[d];
        }
        v += w * (double)A.field[f][off];
      }
      if (f < 2) v = fmin(fmax(v, 0.0), 1.0);
      else if (f == 2) v = fmax(v, 0.0);
    }
    out[(int64_t)f * npts + p] = v;
  }
}

struct VecSet {
  const double* x[kMaxVecs];
};

// partial[i][blk] = sum over this block's cells of x_i * y
__global__ void k_vec_dots(int64_t n, int m, VecSet X, const double* __restrict__ y, double* __restrict__ partial) {
  __shared__ double red[8][kMaxVecs];
  double acc[kMaxVecs];
#pragma unroll
  for (int i = 0; i < kMaxVecs; ++i) acc[i] = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const double yy = y[p];
#pragma unroll
    for (int i = 0; i < kMaxVecs; ++i)
      if (i < m) acc[i] = fma(X.x[i][p], yy, acc[i]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = 0; i < m; ++i) {
    const double v = warp_sum(acc[i]);
    if (lane == 0) red[warp][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < m) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    partial[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void k_vec_reduce(int m, int nblk, const double* __restrict__ partial, double* __restrict__ out) {
  const int i = threadIdx.x;
  if (i >= m) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += partial[(int64_t)i * nblk + b];
  out[i] = s;
}

struct Coefs {
  double c[kMaxVecs];
};

// y may be one of the x_i: each cell is read and written by one thread.
__global__ void k_vec_combine(int64_t n, int m, Coefs C, VecSet X, double beta, double* y) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    double v = beta != 0.0 ? beta * y[p] : 0.0;
    for (int i = 0; i < m; ++i) v = fma(C.c[i], X.x[i][p], v);
    y[p] = v;
  }
}

}  // namespace
}  // namespace orbit

extern "C" {

int orbit_lut_query(const orbit_lut_t* lut, int64_t n_pts, const double* pts, double* out, orbit_stream_t stream) {
  using namespace orbit;
  if (!lut || n_pts < 0 || (n_pts > 0 && (!pts || !out))) {
    set_last_error("orbit_lut_query: bad arguments");
    return ORBIT_ERR_ARG;
  }
  LutArgs A{};
  int64_t s = 1;
  for (int d = kLutDims - 1; d >= 0; --d) {
    if (!lut->axis[d] || lut->n[d] < 2) {
      set_last_error("orbit_lut_query: every axis needs at least two ascending points");
      return ORBIT_ERR_ARG;
    }
    A.axis[d] = lut->axis[d];
    A.n[d] = lut->n[d];
    A.stride[d] = s;
    s *= lut->n[d];
  }
  for (int f = 0; f < 4; ++f) A.field[f] = lut->field[f];
  if (n_pts == 0) return ORBIT_OK;
  cudaStream_t st = (cudaStream_t)stream;
  k_lut_query<<<(unsigned)((n_pts + 127) / 128), 128, 0, st>>>(A, n_pts, pts, out);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

int orbit_vec_dots(int64_t n, int m, const double* const* x, const double* y, double* out, orbit_stream_t stream) {
  using namespace orbit;
  if (n < 1 || m < 1 || m > kMaxVecs || !x || !y || !out) {
    set_last_error("orbit_vec_dots: bad arguments (1 <= m <= 16)");
    return ORBIT_ERR_ARG;
  }
  VecSet X{};
  for (int i = 0; i < m; ++i) {
    if (!x[i]) {
      set_last_error("orbit_vec_dots: null vector");
      return ORBIT_ERR_ARG;
    }
    X.x[i] = x[i];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int nblk = (int)std::min<int64_t>((n + 255) / 256, 296);
  double* scratch = nullptr;
  ORBIT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&scratch), sizeof(double) * ((size_t)m * nblk + m), st));
  k_vec_dots<<<nblk, 256, 0, st>>>(n, m, X, y, scratch);
  note_launch();
  k_vec_reduce<<<1, 32, 0, st>>>(m, nblk, scratch, scratch + (size_t)m * nblk);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch + (size_t)m * nblk, sizeof(double) * m, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(scratch, st);
  if (e != cudaSuccess) {
    set_last_error(std::string("orbit_vec_dots: ") + cudaGetErrorString(e));
    return ORBIT_ERR_CUDA;
  }
  ORBIT_CUDA_TRY(cudaStreamSynchronize(st));
  return ORBIT_OK;
}

int orbit_vec_combine(int64_t n, int m, const double* coef, const double* const* x, double beta, double* y,
                      orbit_stream_t stream) {
  using namespace orbit;
  if (n < 1 || m < 0 || m > kMaxVecs || !y || (m > 0 && (!coef || !x))) {
    set_last_error("orbit_vec_combine: bad arguments (0 <= m <= 16)");
    return ORBIT_ERR_ARG;
  }
  VecSet X{};
  Coefs C{};
  for (int i = 0; i < m; ++i) {
    if (!x[i]) {
      set_last_error("orbit_vec_combine: null vector");
      return ORBIT_ERR_ARG;
    }
    X.x[i] = x[i];
    C.c[i] = coef[i];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int nblk = (int)std::min<int64_t>((n + 255) / 256, 4096);
  k_vec_combine<<<nblk, 256, 0, st>>>(n, m, C, X, beta, y);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

}  // extern "C"
