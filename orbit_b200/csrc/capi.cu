// extern "C" entry points of liborbit_b200 (declared in include/orbit_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <set>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "handles.h"

namespace orbit {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
static std::atomic<long long> g_launches{0};
void note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int allow_max_smem(const void* func) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  ORBIT_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({func, dev})) return ORBIT_OK;
  int optin = 0;
  ORBIT_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  ORBIT_CUDA_TRY(cudaFuncGetAttributes(&fa, func));
  ORBIT_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      optin - (int)fa.sharedSizeBytes));
  done.insert({func, dev});
  return ORBIT_OK;
}

int run_factor(orbit_factor_s* f, int n_active, double dtau, cudaStream_t st);
int launch_chain(orbit_factor_s* f, int B, const int* d_orbit_ids, int trans, int tau0, int tau1,
                 const double* E, double escale, cudaStream_t st);
int orbit_solve_impl(orbit_factor_s* f, int n, const double* e_or_R, double dtau, const double* warm,
                     double tol, int maxiter, int restart, double* out, double* info, int trans,
                     cudaStream_t st);
int chain_apply_impl(orbit_factor_s* f, int n, int trans, int tau0, int tau1, const double* x_in,
                     double* x_out, const double* forcing, double fscale, int refine, cudaStream_t st);
int assemble_transport(int nz, int ny, int nx, const orbit_met_t* met, double* T, double* rowsum,
                       double* lat_loss, cudaStream_t st);
int chain_wait_selftest(orbit_factor_s* f, const int* d_orbit_ids, cudaStream_t st);
int mass_balance_rows(int nz, int ny, int nx, int nbins, const double* const* Tst,
                      const double* const* rho, double* out_int, double* out_top, cudaStream_t st);
int fct_source(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c, double dt,
               int limited, double* d, double* scratch, cudaStream_t st, const double* ghost = nullptr);
int fct_source_noalloc(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c,
                       double dt, int limited, double* d, cudaStream_t st);
int fct_linear_operator(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c, double dt,
                        double* stencil, double* scratch, cudaStream_t st);
int stencil_apply(int nz, int ny, int nx, int px, int n_vec, const double* S, const double* x, double alpha,
                  double beta, int trans, double* y, cudaStream_t st);

namespace {

template <typename T>
int dalloc(std::vector<void*>& allocs, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error(std::string("device allocation of ") + std::to_string(count * sizeof(T)) +
                   " bytes failed: " + cudaGetErrorString(e));
    return ORBIT_ERR_NOMEM;
  }
  allocs.push_back(*p);
  return ORBIT_OK;
}

template <typename T>
int upload(std::vector<void*>& allocs, T** p, const std::vector<T>& v) {
  int rc = dalloc(allocs, p, v.size());
  if (rc) return rc;
  if (!v.empty()) ORBIT_CUDA_TRY(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return ORBIT_OK;
}

void free_all(std::vector<void*>& allocs) {
  for (void* p : allocs) cudaFree(p);
  allocs.clear();
}

#define ORBIT_TRY(expr)        \
  do {                         \
    int _rc = (expr);          \
    if (_rc != ORBIT_OK) {     \
      return _rc;              \
    }                          \
  } while (0)

int build_device_symbolic(orbit_symbolic_s* h) {
  const Symbolic& S = h->S;
  auto& A = h->allocs;
  DevSym& d = h->d;
  ORBIT_TRY(upload(A, &d.first, S.first));
  ORBIT_TRY(upload(A, &d.n, S.n));
  ORBIT_TRY(upload(A, &d.m, S.m));
  ORBIT_TRY(upload(A, &d.parent, S.parent));
  ORBIT_TRY(upload(A, &d.child, S.child));
  ORBIT_TRY(upload(A, &d.uoff, S.uoff));
  ORBIT_TRY(upload(A, &d.uidx, S.uidx));
  ORBIT_TRY(upload(A, &d.rel, S.rel));
  ORBIT_TRY(upload(A, &d.fac_off, S.fac_off));
  ORBIT_TRY(upload(A, &d.ldn, S.ldn));
  ORBIT_TRY(upload(A, &d.ldm, S.ldm));
  ORBIT_TRY(upload(A, &d.ldf, S.ldf));
  ORBIT_TRY(upload(A, &d.front_off, S.front_off));
  ORBIT_TRY(upload(A, &d.woff, S.woff));
  ORBIT_TRY(upload(A, &d.ent_pos, S.ent_pos));
  ORBIT_TRY(upload(A, &d.ent_src, S.ent_src));
  {
    std::vector<int4> fi(S.fitems.size() / 4);
    std::memcpy(fi.data(), S.fitems.data(), fi.size() * sizeof(int4));
    ORBIT_TRY(upload(A, &d.fitems, fi));
  }
  for (int k = 0; k < kNumSched; ++k) {
    const SolveSched& Q = S.sched[k];
    auto& q = d.sched[k];
    std::vector<int4> si(Q.sitems.size() / 4);
    std::memcpy(si.data(), Q.sitems.data(), si.size() * sizeof(int4));
    ORBIT_TRY(upload(A, &q.sitems, si));
    ORBIT_TRY(upload(A, &q.phase_off, Q.phase_off));
    ORBIT_TRY(upload(A, &q.phase_offT, Q.phase_offT));
    ORBIT_TRY(upload(A, &q.nchunk_fwd, Q.nchunk_fwd));
    ORBIT_TRY(upload(A, &q.nchunk_bwd, Q.nchunk_bwd));
    ORBIT_TRY(upload(A, &q.nchunk_fwdT, Q.nchunk_fwdT));
    ORBIT_TRY(upload(A, &q.nchunk_bwdT, Q.nchunk_bwdT));
  }
  ORBIT_TRY(upload(A, &d.perm, S.perm));
  ORBIT_TRY(upload(A, &d.iperm, S.iperm));
  ORBIT_TRY(upload(A, &d.level, S.level));
  ORBIT_TRY(upload(A, &d.tc_pack_off, S.tc_pack_off));
  ORBIT_TRY(upload(A, &d.ginv, S.ginv));
  ORBIT_TRY(upload(A, &d.ginv_off, S.ginv_off));
  return ORBIT_OK;
}

constexpr int kDefaultLeaf = 64;
constexpr int kChunkElems = 8192;

}  // namespace
}  // namespace orbit

using namespace orbit;

extern "C" {

const char* orbit_last_error(void) { return g_last_error.c_str(); }
const char* orbit_version(void) { return "orbit_b200 0.1 (sm_100a)"; }

long long orbit_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int orbit_factor_profile(orbit_factor_t f, int mode, double* out) {
  if (!f) {
    set_last_error("null handle");
    return ORBIT_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(f->mu);
  auto drop = [](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v) {
    for (auto& e : v) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    v.clear();
  };
  if (mode == 0 || mode == 1) {
    drop(f->prof_chain);
    drop(f->prof_factor);
    f->prof_chain_bytes = 0.0;
    f->prof_factor_flops = 0.0;
    f->prof_on = mode == 1;
    return ORBIT_OK;
  }
  if (!out) {
    set_last_error("out is NULL");
    return ORBIT_ERR_ARG;
  }
  auto total = [](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v, double& ms) -> int {
    ms = 0.0;
    for (auto& e : v) {
      ORBIT_CUDA_TRY(cudaEventSynchronize(e.second));
      float t = 0.f;
      ORBIT_CUDA_TRY(cudaEventElapsedTime(&t, e.first, e.second));
      ms += t;
    }
    return ORBIT_OK;
  };
  double cms = 0.0, fms = 0.0;
  int rc = total(f->prof_chain, cms);
  if (rc) return rc;
  rc = total(f->prof_factor, fms);
  if (rc) return rc;
  out[0] = (double)f->prof_chain.size();
  out[1] = cms;
  out[2] = f->prof_chain_bytes;
  out[3] = (double)f->prof_factor.size();
  out[4] = fms;
  out[5] = f->prof_factor_flops;
  return ORBIT_OK;
}

int orbit_symbolic_create_ex(int nz, int ny, int nx, int leaf_cells, int chunk_elems, int tc_min_n,
                             int subtree_div, orbit_symbolic_t* out) {
  return orbit_symbolic_create_grid(nz, ny, nx, 0, leaf_cells, chunk_elems, tc_min_n, subtree_div, out);
}

int orbit_symbolic_create_grid(int nz, int ny, int nx, int periodic_x, int leaf_cells, int chunk_elems,
                               int tc_min_n, int subtree_div, orbit_symbolic_t* out) {
  if (!out) {
    set_last_error("out is NULL");
    return ORBIT_ERR_ARG;
  }
  *out = nullptr;
  // unset options (<= 0; subtree_div < 0) take the environment's value, if
  // any, else the built-in default
  auto env_int = [](const char* name, int fallback) {
    const char* e = std::getenv(name);
    return e ? std::atoi(e) : fallback;
  };
  SymbolicOptions opt;
  opt.leaf_cells = leaf_cells > 0 ? leaf_cells : std::max(1, env_int("ORBIT_B200_LEAF", kDefaultLeaf));
  opt.chunk_elems = std::max(256, chunk_elems > 0 ? chunk_elems : env_int("ORBIT_B200_CHUNK", kChunkElems));
  opt.tc_min_n = std::max(1, tc_min_n > 0 ? tc_min_n : env_int("ORBIT_B200_TC_MIN_N", opt.tc_min_n));
  opt.subtree_div = subtree_div >= 0 ? subtree_div : std::max(0, env_int("ORBIT_B200_SUBTREE_DIV", 0));
  opt.fuse_max_n = std::max(0, env_int("ORBIT_B200_FUSED_MAX_N", kFrontMaxN));
  opt.periodic_x = periodic_x ? 1 : 0;
  orbit_symbolic_s* h = new (std::nothrow) orbit_symbolic_s();
  if (!h) return ORBIT_ERR_NOMEM;
  std::string err = build_symbolic(nz, ny, nx, opt, h->S);
  if (!err.empty()) {
    set_last_error(err);
    delete h;
    return ORBIT_ERR_ARG;
  }
  *out = h;
  return ORBIT_OK;
}

int orbit_symbolic_create(int nz, int ny, int nx, int leaf_cells, orbit_symbolic_t* out) {
  return orbit_symbolic_create_ex(nz, ny, nx, leaf_cells, 0, 0, -1, out);
}

int orbit_symbolic_destroy(orbit_symbolic_t sym) {
  if (!sym) return ORBIT_OK;
  free_all(sym->allocs);
  delete sym;
  return ORBIT_OK;
}

int orbit_symbolic_info(orbit_symbolic_t sym, int64_t* info, int n_info) {
  if (!sym || !info) {
    set_last_error("null argument");
    return ORBIT_ERR_ARG;
  }
  const Symbolic& S = sym->S;
  int64_t v[15] = {S.N, S.nsuper, S.nlevels, S.fac_nnz, S.fac_size, S.front_buf_size, S.max_front,
                   (int64_t)S.factor_flops, S.sched[1].items_per_bin, S.w_size, S.leaf_cells, S.max_nm,
                   S.max_sub_front, S.tc_pack_size, S.n_fused};
  for (int i = 0; i < n_info && i < 15; ++i) info[i] = v[i];
  return ORBIT_OK;
}

int orbit_symbolic_array(orbit_symbolic_t sym, const char* name, void* dst, int64_t capacity,
                         int64_t* count) {
  if (!sym || !name) {
    set_last_error("null argument");
    return ORBIT_ERR_ARG;
  }
  const Symbolic& S = sym->S;
  const void* src = nullptr;
  int64_t cnt = 0;
  size_t es = 4;
  std::string nm(name);
#define ORBIT_ARR(key, vec)                  \
  if (nm == key) {                           \
    src = S.vec.data();                      \
    cnt = (int64_t)S.vec.size();             \
    es = sizeof(S.vec[0]);                   \
  }
  ORBIT_ARR("perm", perm) ORBIT_ARR("iperm", iperm) ORBIT_ARR("first", first) ORBIT_ARR("n", n)
  ORBIT_ARR("m", m) ORBIT_ARR("parent", parent) ORBIT_ARR("level", level) ORBIT_ARR("child", child)
  ORBIT_ARR("uoff", uoff) ORBIT_ARR("uidx", uidx) ORBIT_ARR("rel", rel) ORBIT_ARR("ldn", ldn)
  ORBIT_ARR("ldm", ldm) ORBIT_ARR("ldf", ldf) ORBIT_ARR("fac_off", fac_off)
  ORBIT_ARR("front_off", front_off) ORBIT_ARR("level_front_size", level_front_size)
  ORBIT_ARR("ent_level_off", ent_level_off) ORBIT_ARR("ent_pos", ent_pos) ORBIT_ARR("ent_src", ent_src)
  ORBIT_ARR("ginv", ginv) ORBIT_ARR("ginv_off", ginv_off)
  ORBIT_ARR("woff", woff) ORBIT_ARR("sitems", sched[1].sitems) ORBIT_ARR("phase_off", sched[1].phase_off)
  ORBIT_ARR("phase_offT", sched[1].phase_offT) ORBIT_ARR("nchunk_fwd", sched[1].nchunk_fwd)
  ORBIT_ARR("nchunk_bwd", sched[1].nchunk_bwd) ORBIT_ARR("nchunk_fwdT", sched[1].nchunk_fwdT)
  ORBIT_ARR("nchunk_bwdT", sched[1].nchunk_bwdT)
#undef ORBIT_ARR
  if (!src && cnt == 0 && nm != "sitems") {
    bool known = false;
    for (const char* k : {"perm", "iperm", "first", "n", "m", "parent", "level", "child", "uoff", "uidx",
                          "rel", "ldn", "ldm", "ldf", "fac_off", "front_off", "level_front_size",
                          "ent_level_off", "ent_pos", "ent_src", "ginv", "ginv_off", "woff", "phase_off", "phase_offT",
                          "nchunk_fwd", "nchunk_bwd", "nchunk_fwdT", "nchunk_bwdT"})
      known = known || nm == k;
    if (!known) {
      set_last_error("unknown symbolic array " + nm);
      return ORBIT_ERR_ARG;
    }
  }
  if (count) *count = cnt;
  if (dst) {
    if (capacity < cnt) {
      set_last_error("destination too small");
      return ORBIT_ERR_ARG;
    }
    if (cnt) std::memcpy(dst, src, (size_t)cnt * es);
  }
  return ORBIT_OK;
}

int orbit_symbolic_perm(orbit_symbolic_t sym, int32_t* perm_host) {
  if (!sym || !perm_host) {
    set_last_error("null argument");
    return ORBIT_ERR_ARG;
  }
  std::memcpy(perm_host, sym->S.perm.data(), sym->S.perm.size() * sizeof(int32_t));
  return ORBIT_OK;
}

int orbit_assemble_transport(int nz, int ny, int nx, const orbit_met_t* met, double* T_stencil,
                             double* rowsum, orbit_stream_t stream) {
  if (!met || !T_stencil || nz < 1 || ny < 2 || nx < 2) {
    set_last_error("orbit_assemble_transport: bad arguments (need nz>=1, ny>=2, nx>=2)");
    return ORBIT_ERR_ARG;
  }
  if (!met->dP || !met->Dz || !met->u || !met->v || !met->kxxyy || !met->kzz || !met->w_plus ||
      !met->w_minus || !met->lat || (met->split && (!met->u_plus || !met->u_minus || !met->v_plus ||
                                                    !met->v_minus || !met->u_plus_e || !met->v_plus_n)) ||
      (!met->split && (!met->u_e || !met->v_n))) {
    set_last_error("orbit_assemble_transport: missing meteorology field");
    return ORBIT_ERR_ARG;
  }
  if (met->periodic_lon && (nx < 3 || !met->u_wrap || (met->split && (!met->u_plus_wrap || !met->u_minus_wrap)))) {
    set_last_error("orbit_assemble_transport: a periodic-longitude grid needs nx >= 3 and the wrap-face fields");
    return ORBIT_ERR_ARG;
  }
  return assemble_transport(nz, ny, nx, met, T_stencil, rowsum, nullptr, (cudaStream_t)stream);
}

int orbit_transport_boundary_loss(int nz, int ny, int nx, const orbit_met_t* met, double* loss,
                                  orbit_stream_t stream) {
  if (!met || !loss || nz < 1 || ny < 2 || nx < 2) {
    set_last_error("orbit_transport_boundary_loss: bad arguments (need nz>=1, ny>=2, nx>=2)");
    return ORBIT_ERR_ARG;
  }
  if (!met->dP || !met->Dz || !met->u || !met->v || !met->kxxyy || !met->kzz || !met->w_plus ||
      !met->w_minus || !met->lat || (met->split && (!met->u_minus || !met->v_minus || !met->u_plus_e ||
                                                    !met->v_plus_n)) ||
      (!met->split && (!met->u_e || !met->v_n))) {
    set_last_error("orbit_transport_boundary_loss: missing meteorology field");
    return ORBIT_ERR_ARG;
  }
  return assemble_transport(nz, ny, nx, met, nullptr, nullptr, loss, (cudaStream_t)stream);
}

int orbit_mass_balance_rows(int nz, int ny, int nx, int nbins, const double* const* T_stencils,
                            const double* const* rho, double* out_interior, double* out_top,
                            orbit_stream_t stream) {
  if (nbins < 1 || ny < 3 || nx < 3 || !T_stencils || !rho || !out_interior || !out_top) {
    set_last_error("orbit_mass_balance_rows: bad arguments");
    return ORBIT_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const double** d = nullptr;
  ORBIT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(double*) * 2 * nbins, st));
  ORBIT_CUDA_TRY(cudaMemcpyAsync(d, T_stencils, sizeof(double*) * nbins, cudaMemcpyHostToDevice, st));
  ORBIT_CUDA_TRY(cudaMemcpyAsync(d + nbins, rho, sizeof(double*) * nbins, cudaMemcpyHostToDevice, st));
  int rc = mass_balance_rows(nz, ny, nx, nbins, d, d + nbins, out_interior, out_top, st);
  cudaFreeAsync(d, st);
  ORBIT_CUDA_TRY(cudaStreamSynchronize(st));
  return rc;
}

int orbit_fct_source(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c, double dt,
                     int limited, double* d, orbit_stream_t stream) {
  if (!met || !c || !d || n_vec < 1 || nz < 1 || ny < 1 || nx < 1 || !(dt > 0)) {
    set_last_error("orbit_fct_source: bad arguments");
    return ORBIT_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t N = (int64_t)nz * ny * nx;
  double* scratch = nullptr;
  ORBIT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&scratch), sizeof(double) * 3 * N * n_vec, st));
  int rc = fct_source(nz, ny, nx, met, n_vec, c, dt, limited, d, scratch, st);
  cudaFreeAsync(scratch, st);
  return rc;
}

int orbit_fct_linear_operator(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c_base,
                              double dt, double* stencil, orbit_stream_t stream) {
  if (!met || !c_base || !stencil || n_vec < 1 || nz < 1 || ny < 1 || nx < 1 || !(dt > 0)) {
    set_last_error("orbit_fct_linear_operator: bad arguments");
    return ORBIT_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t N = (int64_t)nz * ny * nx;
  double* scratch = nullptr;
  ORBIT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&scratch), sizeof(double) * 3 * N * n_vec, st));
  int rc = fct_linear_operator(nz, ny, nx, met, n_vec, c_base, dt, stencil, scratch, st);
  cudaFreeAsync(scratch, st);
  return rc;
}

int orbit_fct_source_ghost(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c,
                           const double* c_ghost, double dt, int limited, double* d, orbit_stream_t stream) {
  if (!met || !c || !c_ghost || !d || n_vec < 1 || nz < 1 || ny < 1 || nx < 1 || !(dt > 0)) {
    set_last_error("orbit_fct_source_ghost: bad arguments");
    return ORBIT_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t N = (int64_t)nz * ny * nx;
  double* scratch = nullptr;
  ORBIT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&scratch), sizeof(double) * 3 * N * n_vec, st));
  int rc = fct_source(nz, ny, nx, met, n_vec, c, dt, limited, d, scratch, st, c_ghost);
  cudaFreeAsync(scratch, st);
  return rc;
}

int orbit_stencil_apply(int nz, int ny, int nx, int n_vec, const double* stencils, const double* x, double alpha,
                        double beta, int trans, double* y, orbit_stream_t stream) {
  if (!stencils || !x || !y || n_vec < 1 || nz < 1 || ny < 1 || nx < 1) {
    set_last_error("orbit_stencil_apply: bad arguments");
    return ORBIT_ERR_ARG;
  }
  return stencil_apply(nz, ny, nx, 0, n_vec, stencils, x, alpha, beta, trans, y, (cudaStream_t)stream);
}

int orbit_stencil_apply_grid(int nz, int ny, int nx, int periodic_x, int n_vec, const double* stencils,
                             const double* x, double alpha, double beta, int trans, double* y,
                             orbit_stream_t stream) {
  if (!stencils || !x || !y || n_vec < 1 || nz < 1 || ny < 1 || nx < 1 || (periodic_x && nx < 3)) {
    set_last_error("orbit_stencil_apply_grid: bad arguments");
    return ORBIT_ERR_ARG;
  }
  return stencil_apply(nz, ny, nx, periodic_x ? 1 : 0, n_vec, stencils, x, alpha, beta, trans, y,
                       (cudaStream_t)stream);
}

int orbit_fct_source_noalloc(int nz, int ny, int nx, const orbit_met_t* met, int n_vec, const double* c,
                             double dt, int limited, double* d, orbit_stream_t stream) {
  if (!met || !c || !d || n_vec < 1 || nz < 1 || ny < 1 || nx < 1 || !(dt > 0)) {
    set_last_error("orbit_fct_source_noalloc: bad arguments");
    return ORBIT_ERR_ARG;
  }
  return fct_source_noalloc(nz, ny, nx, met, n_vec, c, dt, limited, d, (cudaStream_t)stream);
}

int orbit_factor_create_ex(orbit_symbolic_t sym, int n_orbits, int n_sets, int n_bins, int precision,
                           orbit_factor_t* out) {
  if (!sym || !out || n_orbits < 1 || n_sets < 1 || (n_bins != 1 && n_bins != 8) ||
      (n_bins == 1 && (n_orbits != 1 || n_sets != 1)) ||
      (precision != ORBIT_PREC_FP64 && precision != ORBIT_PREC_FP32)) {
    set_last_error("orbit_factor_create_ex: bad arguments (n_bins is 8, or 1 with one orbit and one set)");
    return ORBIT_ERR_ARG;
  }
  *out = nullptr;
  {
    // device copies of the symbolic arrays are made on first use
    std::lock_guard<std::mutex> lk(sym->mu);
    if (!sym->uploaded) {
      int rc0 = build_device_symbolic(sym);
      if (rc0) {
        free_all(sym->allocs);
        sym->d = DevSym();
        return rc0;
      }
      cudaGetDevice(&sym->device);
      sym->uploaded = true;
    }
  }
  orbit_factor_s* f = new (std::nothrow) orbit_factor_s();
  if (!f) return ORBIT_ERR_NOMEM;
  f->sym = sym;
  f->n_orbits = n_orbits;
  f->n_sets = n_sets;
  f->n_bins = n_bins;
  f->precision = precision;
  cudaGetDevice(&f->device);
  const Symbolic& S = sym->S;
  const int64_t N = S.N;
  const size_t vb = precision == ORBIT_PREC_FP32 ? 4 : 8;
  const int64_t n_inst = (int64_t)n_sets * n_bins;
  auto& A = f->allocs;
  int rc = ORBIT_OK;
  auto fail = [&](int code) {
    free_all(A);
    delete f;
    return code;
  };
  // fronts: group size from a budget
  // Factorization scratch (two level buffers of fronts per instance, plus the
  // tensor-core operand packs of fp32 factors) for a group of instances that
  // is factored together: 48 GB or a quarter of the device, whichever is
  // smaller, with the instances split into groups of equal size.
  size_t budget = (size_t)48 << 30;
  {
    int dev = 0;
    size_t free_b = 0, total_b = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && total_b > 0)
      budget = std::min(budget, total_b / 4);
    else
      cudaGetLastError();
  }
  if (const char* e = std::getenv("ORBIT_B200_FRONT_BUDGET_GB")) budget = (size_t)(std::atof(e) * (1 << 30));
  const int64_t per_inst =
      2 * S.front_buf_size * (int64_t)vb + (precision == ORBIT_PREC_FP32 ? S.tc_pack_size * 4 : 0);
  int64_t G = per_inst > 0 ? std::max<int64_t>(1, (int64_t)(budget / per_inst)) : n_inst;
  G = std::min<int64_t>(G, n_inst);
  const int64_t ngroups = (n_inst + G - 1) / G;
  G = (n_inst + ngroups - 1) / ngroups;
  f->front_group = (int)G;
  if ((rc = dalloc(A, reinterpret_cast<unsigned char**>(&f->factors), (size_t)n_inst * S.fac_size * vb))) return fail(rc);
  if ((rc = dalloc(A, reinterpret_cast<unsigned char**>(&f->fronts), (size_t)2 * G * S.front_buf_size * vb))) return fail(rc);
  if (precision == ORBIT_PREC_FP32 && S.tc_pack_size > 0)
    if ((rc = dalloc(A, &f->tc_pack, (size_t)G * S.tc_pack_size))) return fail(rc);
  if ((rc = dalloc(A, &f->A_stencil, (size_t)n_inst * 7 * N))) return fail(rc);
  if ((rc = dalloc(A, &f->d_Tptr, (size_t)n_inst))) return fail(rc);
  if ((rc = dalloc(A, &f->d_Dptr, (size_t)n_inst))) return fail(rc);
  if ((rc = dalloc(A, &f->X, (size_t)n_orbits * 9 * N))) return fail(rc);
  if ((rc = dalloc(A, &f->Ybuf, (size_t)n_orbits * N))) return fail(rc);
  if ((rc = dalloc(A, &f->Wbuf, (size_t)n_orbits * S.w_size))) return fail(rc);
  if ((rc = dalloc(A, &f->counters, (size_t)n_orbits * 16 * S.nsuper))) return fail(rc);
  if ((rc = dalloc(A, &f->E, (size_t)n_orbits * 8 * N))) return fail(rc);
  if ((rc = dalloc(A, &f->tmpv, (size_t)n_orbits * 23 * N))) return fail(rc);
  if ((rc = dalloc(A, &f->orbit_ids, (size_t)n_orbits))) return fail(rc);
  if ((rc = dalloc(A, &f->set_of, (size_t)n_orbits))) return fail(rc);
  f->h_set_of.resize(n_orbits);
  for (int o = 0; o < n_orbits; ++o) f->h_set_of[o] = o % n_sets;
  if (cudaMemcpy(f->set_of, f->h_set_of.data(), sizeof(int) * n_orbits, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(ORBIT_ERR_CUDA);
  if ((rc = dalloc(A, &f->task_counter, (size_t)1 + n_orbits))) return fail(rc);
  if ((rc = dalloc(A, &f->status, (size_t)1))) return fail(rc);
  f->restart_cap = 31;
  if ((rc = dalloc(A, &f->V, (size_t)n_orbits * 33 * N))) return fail(rc);
  if ((rc = dalloc(A, &f->Hd, (size_t)n_orbits * 33 * 32))) return fail(rc);
  if ((rc = dalloc(A, &f->gv, (size_t)n_orbits * 33))) return fail(rc);
  if ((rc = dalloc(A, &f->cs, (size_t)n_orbits * 32))) return fail(rc);
  if ((rc = dalloc(A, &f->sn, (size_t)n_orbits * 32))) return fail(rc);
  if ((rc = dalloc(A, &f->red, (size_t)n_orbits * 33 + (size_t)n_orbits * 32 * 33 * 48))) return fail(rc);
  if ((rc = dalloc(A, &f->scal, (size_t)n_orbits * 16))) return fail(rc);
  if (cudaMallocHost(reinterpret_cast<void**>(&f->h_status), sizeof(int)) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void**>(&f->h_scal), sizeof(double) * 16 * n_orbits) != cudaSuccess) {
    cudaGetLastError();
    set_last_error("pinned host allocation failed");
    return fail(ORBIT_ERR_NOMEM);
  }
  if (cudaMemset(f->status, 0, sizeof(int)) != cudaSuccess) return fail(ORBIT_ERR_CUDA);
  *out = f;
  return ORBIT_OK;
}

int orbit_factor_create(orbit_symbolic_t sym, int n_orbits, int precision, orbit_factor_t* out) {
  return orbit_factor_create_ex(sym, n_orbits, n_orbits, 8, precision, out);
}

int orbit_factor_map(orbit_factor_t f, const int32_t* set_of_orbit) {
  if (!f || !set_of_orbit) {
    set_last_error("orbit_factor_map: null argument");
    return ORBIT_ERR_ARG;
  }
  for (int o = 0; o < f->n_orbits; ++o)
    if (set_of_orbit[o] < 0 || set_of_orbit[o] >= f->n_sets) {
      set_last_error("orbit_factor_map: factor set index out of range");
      return ORBIT_ERR_ARG;
    }
  std::lock_guard<std::mutex> lk(f->mu);
  f->h_set_of.assign(set_of_orbit, set_of_orbit + f->n_orbits);
  ORBIT_CUDA_TRY(cudaMemcpy(f->set_of, f->h_set_of.data(), sizeof(int) * f->n_orbits, cudaMemcpyHostToDevice));
  return ORBIT_OK;
}

int orbit_factor_destroy(orbit_factor_t f) {
  if (!f) return ORBIT_OK;
  cudaDeviceSynchronize();
  orbit_factor_profile(f, 0, nullptr);
  free_all(f->allocs);
  if (f->h_status) cudaFreeHost(f->h_status);
  if (f->h_scal) cudaFreeHost(f->h_scal);
  delete f;
  return ORBIT_OK;
}

int orbit_factor_numeric(orbit_factor_t f, int n_active, const double* const* T_stencils,
                         const double* const* sink_diags, double dtau, orbit_stream_t stream) {
  if (!f || !T_stencils || n_active < 1 || n_active > f->n_sets || !(dtau > 0)) {
    set_last_error("orbit_factor_numeric: bad arguments (n_active factor sets <= n_sets)");
    return ORBIT_ERR_ARG;
  }
  const int nb = f->n_bins;
  for (int i = 0; i < n_active * nb; ++i)
    if (!T_stencils[i]) {
      set_last_error("orbit_factor_numeric: NULL transport stencil");
      return ORBIT_ERR_ARG;
    }
  std::lock_guard<std::mutex> lk(f->mu);
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<const double*> dp(n_active * nb, nullptr);
  if (sink_diags)
    for (int i = 0; i < n_active * nb; ++i) dp[i] = sink_diags[i];
  ORBIT_CUDA_TRY(cudaMemcpyAsync(f->d_Tptr, T_stencils, sizeof(double*) * n_active * nb, cudaMemcpyHostToDevice, st));
  ORBIT_CUDA_TRY(cudaMemcpyAsync(f->d_Dptr, dp.data(), sizeof(double*) * n_active * nb, cudaMemcpyHostToDevice, st));
  ORBIT_CUDA_TRY(cudaMemsetAsync(f->status, 0, sizeof(int), st));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (f->prof_on) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
  }
  int rc = run_factor(f, n_active, dtau, st);
  if (f->prof_on) {
    cudaEventRecord(e1, st);
    f->prof_factor.push_back({e0, e1});
    f->prof_factor_flops += (double)n_active * nb * f->sym->S.factor_flops;
  }
  if (rc) return rc;
  ORBIT_CUDA_TRY(cudaMemcpyAsync(f->h_status, f->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  ORBIT_CUDA_TRY(cudaStreamSynchronize(st));
  if (*f->h_status != 0) {
    set_last_error(*f->h_status == ORBIT_ERR_TIMEOUT
                       ? "tensor-core Schur complement: a pipeline wait exceeded its limit"
                       : "zero or non-finite pivot in the numeric factorization");
    return *f->h_status;
  }
  f->n_factored = n_active;
  f->dtau = dtau;
  return ORBIT_OK;
}

int orbit_factor_bytes(orbit_factor_t f, int64_t* numeric_bytes, int64_t* workspace_bytes) {
  if (!f) {
    set_last_error("null handle");
    return ORBIT_ERR_ARG;
  }
  const Symbolic& S = f->sym->S;
  const int64_t vb = f->precision == ORBIT_PREC_FP32 ? 4 : 8;
  if (numeric_bytes) *numeric_bytes = (int64_t)f->n_sets * f->n_bins * S.fac_size * vb;
  if (workspace_bytes)
    *workspace_bytes = (int64_t)2 * f->front_group * S.front_buf_size * vb +
                       (f->tc_pack ? (int64_t)f->front_group * S.tc_pack_size * 4 : 0) +
                       (int64_t)f->n_sets * f->n_bins * 7 * S.N * 8 +
                       (int64_t)f->n_orbits * (9 + 1 + 8 + 23 + 33) * S.N * 8;
  return ORBIT_OK;
}

static int check_slots(orbit_factor_t f, int n_active, bool need_8_bins) {
  if (need_8_bins && f->n_bins != 8) {
    set_last_error("periodic-orbit solves need an 8-bin factor handle");
    return ORBIT_ERR_ARG;
  }
  if (n_active < 1 || n_active > f->n_orbits) {
    set_last_error("n_active out of range");
    return ORBIT_ERR_ARG;
  }
  for (int o = 0; o < n_active; ++o)
    if (f->h_set_of[o] >= f->n_factored) {
      set_last_error("an active orbit maps to a factor set that has not been factored");
      return ORBIT_ERR_ARG;
    }
  return ORBIT_OK;
}

int orbit_chain_apply(orbit_factor_t f, int n_active, int trans, int tau0, int tau1, const double* x_in,
                      double* x_out, const double* forcing, double fscale, int refine,
                      orbit_stream_t stream) {
  if (!f || !x_in || !x_out || tau0 < 0 || tau1 > f->n_bins || tau0 >= tau1) {
    set_last_error("orbit_chain_apply: bad arguments (0 <= tau0 < tau1 <= bins of the handle)");
    return ORBIT_ERR_ARG;
  }
  if (int rc0 = check_slots(f, n_active, false)) return rc0;
  std::lock_guard<std::mutex> lk(f->mu);
  return chain_apply_impl(f, n_active, trans, tau0, tau1, x_in, x_out, forcing, fscale, refine,
                          (cudaStream_t)stream);
}

int orbit_selftest_wait_timeout(orbit_factor_t f, orbit_stream_t stream) {
  if (!f || f->n_factored < 1) {
    set_last_error("orbit_selftest_wait_timeout: factor the handle first");
    return ORBIT_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(f->mu);
  cudaStream_t st = (cudaStream_t)stream;
  const int zero = 0;
  ORBIT_CUDA_TRY(cudaMemcpyAsync(f->orbit_ids, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
  int rc = chain_wait_selftest(f, f->orbit_ids, st);
  if (rc == ORBIT_ERR_TIMEOUT) set_last_error("device spin-wait timed out (self-test)");
  return rc;
}

int orbit_gmres_solve(orbit_factor_t f, int n_active, const double* e, double dtau, const double* c_warm,
                      double tol, int maxiter, int restart, double* orbit_out, double* info_out,
                      orbit_stream_t stream) {
  if (!f || !e || !orbit_out || !info_out || !(tol > 0) || maxiter < 1) {
    set_last_error("orbit_gmres_solve: bad arguments");
    return ORBIT_ERR_ARG;
  }
  if (int rc0 = check_slots(f, n_active, true)) return rc0;
  std::lock_guard<std::mutex> lk(f->mu);
  return orbit_solve_impl(f, n_active, e, dtau, c_warm, tol, maxiter, restart, orbit_out, info_out, 0,
                          (cudaStream_t)stream);
}

int orbit_adjoint_gmres_solve(orbit_factor_t f, int n_active, const double* R, const double* lam_warm,
                              double tol, int maxiter, int restart, double* adjoint_out, double* info_out,
                              orbit_stream_t stream) {
  if (!f || !R || !adjoint_out || !info_out || !(tol > 0) || maxiter < 1) {
    set_last_error("orbit_adjoint_gmres_solve: bad arguments");
    return ORBIT_ERR_ARG;
  }
  if (int rc0 = check_slots(f, n_active, true)) return rc0;
  std::lock_guard<std::mutex> lk(f->mu);
  return orbit_solve_impl(f, n_active, R, 1.0, lam_warm, tol, maxiter, restart, adjoint_out, info_out, 1,
                          (cudaStream_t)stream);
}

}  // extern "C"
