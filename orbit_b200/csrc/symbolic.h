// Host symbolic analysis for the 7-point operator I + dtau L on an
// (nz, ny, nx) box: geometric nested dissection into dense supernodes, the
// multifrontal extend-add maps, and the static launch schedules of the
// numeric factorization and of the chained triangular solves.
//
// One symbolic serves every species, bin and met draw of a domain shape: the
// matrix pattern is the full 7-point stencil (explicit zeros where a face
// carries no flux), which is the pattern-reuse contract the reference relies
// on when it hands one UMFPACK symbolic to every species
// (orbit/core/solve.py:88-207, orbit/core/orbit.py:79-96).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace orbit {

// Stencil directions of the 7-point operator; values live as
// stencil[dir * N + cell], cell = k*ny*nx + j*nx + i (reference CellIndexer,
// orbit/core/indexing.py:5-45).
enum StencilDir { D_C = 0, D_W = 1, D_E = 2, D_S = 3, D_N = 4, D_B = 5, D_T = 6 };

constexpr int kTile = 64;      // dense tile edge of the factorization kernels
constexpr int kNB = 64;        // panel width of the blocked LU
constexpr int kPad = 4;        // leading-dimension padding (elements)
constexpr int kSchurTile = 128;  // output tile edge of the Schur-complement GEMM
constexpr int kTcK = 16;         // K extent of one packed tensor-core operand tile
constexpr int kTcTileFloats = kSchurTile * kTcK;  // floats per packed plane
constexpr int kTcPackRun = 4;        // k-blocks of one operand row tile packed by one CTA
constexpr int kFrontMaxN = 64;        // largest pivot count of a one-CTA front
constexpr int kFrontMaxElems = 28672;  // its shared-memory budget in elements (224 KB of FP64)

// Shared-memory elements of a one-CTA front (k_front): the pivot block's
// inverses and their transpose (n x ldq each), both panels (n x ldl each)
// and the pivot steps' exchange slots (2 x 4 x 64).
inline int64_t front_smem_elems(int64_t n, int64_t m) {
  const int64_t ldq = (n + 3) / 4 * 4 + 4, ldl = (m + 3) / 4 * 4;
  return 2 * n * ldq + 2 * n * ldl + 512;
}

inline int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

// One kernel launch of the numeric factorization schedule.
struct FactorLaunch {
  enum Kind : int { ZERO = 0, SCATTER, EXTEND, DIAG, PANEL, UPDATE, SCHUR, INV, TRIL, PRODL, TRIU, PRODU, TC_PACK, ASSEMBLE, TC_GEMM, FRONT } kind;
  int level;
  int p0;          // pivot-block start (DIAG/PANEL/UPDATE/INV); SCHUR: leading items of CUDA-core nodes;
                   // FRONT: shared-memory elements of the largest front in the launch
  int64_t item_off;  // offset into the item array (int4 units)
  int64_t items;     // number of items (per instance)
};

// Solve schedule (per bin, shared by all instances): items {s, r0, r1, kind}
// with kinds 0 fwd, 1 bwd, 2 fwdT, 3 bwdT (row chunks of one supernode) and
// 4..7 the same sweeps over a whole subtree {root, first node, 0, kind}.
struct SolveSched {
  int chunk_elems = 0;
  std::vector<int32_t> sitems;            // 4 ints per item
  std::vector<int32_t> phase_off;         // non-transposed phases (2*nlevels+1 offsets)
  std::vector<int32_t> phase_offT;        // transposed phases
  int32_t items_per_bin = 0, items_per_binT = 0;
  // per supernode number of chunks in each solve kind
  std::vector<int32_t> nchunk_fwd, nchunk_bwd, nchunk_fwdT, nchunk_bwdT;
};
constexpr int kNumSched = 3;

struct Symbolic {
  int nz = 0, ny = 0, nx = 0;
  int periodic_x = 0;  // periodic longitude: columns i = 0 and i = nx - 1 are neighbours
  int64_t N = 0;
  int leaf_cells = 0;
  int nsuper = 0;
  int nlevels = 0;
  // permutation: perm[new] = old cell; iperm[old] = new
  std::vector<int32_t> perm, iperm;
  // per supernode (postorder = elimination order)
  std::vector<int32_t> first, n, m, parent, level, nchild;
  std::vector<int32_t> child;        // 2 per supernode (-1 = none)
  std::vector<int64_t> uoff;         // offset into uidx/rel, size nsuper+1
  std::vector<int32_t> uidx;         // ancestor unknowns (new index), sorted
  std::vector<int32_t> rel;          // position of uidx[i] in the parent front
  std::vector<int32_t> sup_of;       // new index -> owning supernode
  // dense storage
  std::vector<int32_t> ldn, ldm, ldf;     // leading dims (padded)
  std::vector<int64_t> fac_off;           // factor block offset per supernode
  int64_t fac_size = 0;                   // elements per factor instance
  int64_t fac_nnz = 0;                    // structural nonzeros sum(n^2 + 2nm)
  std::vector<int64_t> front_off;         // offset within its level buffer
  std::vector<int64_t> level_front_size;  // elements per instance per level
  int64_t front_buf_size = 0;             // max over levels of level_front_size
  std::vector<int64_t> woff;              // update-vector offset per supernode
  // inverse extend-add maps: for supernode s, 2 x (n+m) ints at ginv_off[s];
  // entry [q][i] is the update index u of child q with rel_c[u] == i, or -1
  std::vector<int32_t> ginv;
  std::vector<int64_t> ginv_off;
  int64_t w_size = 0;
  // per level: supernodes of that level
  std::vector<std::vector<int32_t>> level_sups;
  // original-entry scatter: per level, (front position, stencil index) pairs
  std::vector<int64_t> ent_level_off;     // size nlevels+1
  std::vector<int64_t> ent_pos;           // position within the front (row*ld+col) + front_off
  std::vector<int32_t> ent_src;           // dir*N + cell
  // factorization schedule; items are int4 {a,b,c,d}
  std::vector<int32_t> fitems;            // 4 ints per item
  std::vector<FactorLaunch> fsched;
  SolveSched sched[kNumSched];  // chunk/2, chunk, 2 chunk; sched[1] is the default
  std::vector<int32_t> role;  // 0 chunked node, 1 subtree-task root, 2 inside a subtree
  int max_front = 0;
  int max_sub_front = 0;  // largest n+m of a supernode inside a subtree task
  int max_nm = 0;
  double factor_flops = 0.0;
  // tensor-core pipeline (fp32 factors) for supernodes with n >= tc_min_n and
  // m > 0: tc_pack_off[s] is the float offset of the node's tf32 hi/lo operand
  // tiles inside its level's per-instance pack buffer, -1 for other nodes.
  int tc_min_n = 0;
  std::vector<int64_t> tc_pack_off;
  int64_t tc_pack_size = 0;  // floats per instance (max over levels)
  // one-CTA fronts: supernodes with 0 < n <= fuse_max_n, m > 0 and
  // front_smem_elems(n, m) <= kFrontMaxElems are factored whole by one CTA
  int fuse_max_n = 0;
  int64_t n_fused = 0;
};

// Tuning options of the analysis (the autotuner's search space).
struct SymbolicOptions {
  int leaf_cells = 64;    // nested-dissection leaf size (cells)
  int chunk_elems = 8192; // solve row-chunk size of the medium schedule (factor entries)
  int tc_min_n = 48;      // smallest pivot count of a tensor-core supernode (fp32 factors)
  int subtree_div = 0;    // > 0: whole-subtree solve tasks below fac_nnz / subtree_div; 0: none
  int fuse_max_n = kFrontMaxN;  // largest pivot count of a one-CTA front (0: none)
  int periodic_x = 0;     // periodic longitude (needs nx >= 3)
};

// Build the symbolic analysis.  Returns an empty string on success, an
// error message otherwise.
std::string build_symbolic(int nz, int ny, int nx, const SymbolicOptions& opt, Symbolic& S);

}  // namespace orbit
