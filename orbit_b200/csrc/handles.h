// Internal layout of the opaque handles of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "symbolic.h"

struct DevSym {
  // device copies of the symbolic arrays
  int32_t *first = nullptr, *n = nullptr, *m = nullptr, *parent = nullptr, *child = nullptr;
  int64_t *uoff = nullptr;
  int32_t *uidx = nullptr, *rel = nullptr;
  int64_t *fac_off = nullptr;
  int32_t *ldn = nullptr, *ldm = nullptr, *ldf = nullptr;
  int64_t *front_off = nullptr, *woff = nullptr;
  int64_t *ent_pos = nullptr;
  int32_t *ent_src = nullptr;
  int4 *fitems = nullptr;
  struct Sched {
    int4 *sitems = nullptr;
    int32_t *phase_off = nullptr, *phase_offT = nullptr;
    int32_t *nchunk_fwd = nullptr, *nchunk_bwd = nullptr, *nchunk_fwdT = nullptr, *nchunk_bwdT = nullptr;
  } sched[orbit::kNumSched];
  int32_t *perm = nullptr, *iperm = nullptr;
  int32_t *level = nullptr;
  int64_t *tc_pack_off = nullptr;
  int32_t *ginv = nullptr;
  int64_t *ginv_off = nullptr;
};

struct orbit_symbolic_s {
  orbit::Symbolic S;
  DevSym d;
  int device = 0;
  bool uploaded = false;
  std::mutex mu;
  std::vector<void*> allocs;
};

struct orbit_factor_s {
  orbit_symbolic_s* sym = nullptr;
  int n_orbits = 0;   // solve slots (vectors, counters)
  int n_sets = 0;     // factor sets (each n_bins factorizations)
  int n_bins = 8;     // 8, or 1 for a single-factor handle
  int* set_of = nullptr;           // device: factor set of each solve slot
  std::vector<int> h_set_of;       // host mirror
  int precision = 64;
  int device = 0;
  int n_factored = 0;
  double dtau = 10800.0;
  // factor values: (n_orbits * 8) instances of fac_size elements (T = double or float)
  void* factors = nullptr;
  // front workspace: 2 parity buffers x group instances x front_buf_size
  void* fronts = nullptr;
  int front_group = 1;
  // fp32 factors: tf32 hi/lo operand packs of the tensor-core Schur
  // complements, front_group instances x tc_pack_size floats
  float* tc_pack = nullptr;
  // FP64 copies of A = I + dtau (T + diag(sink)) as 7-point stencils, per instance
  double* A_stencil = nullptr;
  // device pointer tables (per instance) used by the scatter kernel
  const double** d_Tptr = nullptr;
  const double** d_Dptr = nullptr;
  // solve workspace (per orbit)
  double* X = nullptr;      // 9 N (new order)
  double* Ybuf = nullptr;   // N
  double* Wbuf = nullptr;   // w_size
  int* counters = nullptr;  // 8 * 2 * nsuper
  double* E = nullptr;      // 8 N forcing (new order)
  double* tmpv = nullptr;   // 4 N scratch vectors
  int* orbit_ids = nullptr; // n_orbits
  int* task_counter = nullptr;
  int* status = nullptr;    // device status word
  int* h_status = nullptr;  // pinned
  // GMRES workspace
  int restart_cap = 0;
  double* V = nullptr;      // (restart+1) N per orbit
  double* Hd = nullptr;     // per orbit (restart+1)*restart
  double* gv = nullptr;     // per orbit restart+1 (g), cs, sn
  double* cs = nullptr;
  double* sn = nullptr;
  double* red = nullptr;    // reduction scratch
  double* scal = nullptr;   // per orbit scalars
  double* h_scal = nullptr; // pinned mirror
  int persist_grid = 0;
  // optional per-launch timing of the chain kernel and of factorizations
  bool prof_on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_chain, prof_factor;
  double prof_chain_bytes = 0.0, prof_factor_flops = 0.0;
  std::mutex mu;
  std::vector<void*> allocs;
};
