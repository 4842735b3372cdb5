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
