// Shared device helpers and status codes of liborbit_b200.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "../../include/orbit_b200.h"

namespace orbit {

void set_last_error(const std::string& msg);
// Count of kernels this library has launched (all handles, all threads).
void note_launch(int n = 1);
// Raise a kernel's dynamic shared-memory limit to the device's opt-in maximum,
// once per (kernel, device).  The limit is per-function state shared by every
// thread, so it is only ever raised, never set per call.
int allow_max_smem(const void* func);

#define ORBIT_CUDA_TRY(expr)                                                     \
  do {                                                                           \
    cudaError_t _e = (expr);                                                     \
    if (_e != cudaSuccess) {                                                     \
      ::orbit::set_last_error(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
      return ORBIT_ERR_CUDA;                                                     \
    }                                                                            \
  } while (0)

// Neighbours of cell c of an (nz, ny, nx) grid in the stencil order W E S N
// B T, and whether each exists.  With px set (periodic longitude, nx >= 3)
// the x neighbours of the first and last columns wrap around: the stencil's
// W entry of a cell with i = 0 couples it to i = nx - 1 and the E entry of
// i = nx - 1 to i = 0 (orbit/core/convdiff.py:150-202).
__device__ __forceinline__ void stencil_nbrs(int64_t c, int nz, int ny, int nx, int px, int64_t nb[6],
                                             bool has[6]) {
  const int64_t nxy = (int64_t)nx * ny;
  const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / nxy);
  nb[0] = i > 0 ? c - 1 : c + nx - 1;
  nb[1] = i < nx - 1 ? c + 1 : c - (nx - 1);
  nb[2] = c - nx;
  nb[3] = c + nx;
  nb[4] = c - nxy;
  nb[5] = c + nxy;
  has[0] = i > 0 || px;
  has[1] = i < nx - 1 || px;
  has[2] = j > 0;
  has[3] = j < ny - 1;
  has[4] = k > 0;
  has[5] = k < nz - 1;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile(const int* p) {
  return *reinterpret_cast<const volatile int*>(p);
}

__device__ __forceinline__ void raise_status(int* status, int code) {
  atomicCAS(status, 0, code);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace orbit
