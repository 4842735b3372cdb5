// Geometric nested dissection + dense-supernode symbolic analysis.
//
// The reference factors each I + dtau L_tau with UMFPACK (or SuperLU) behind
// a fill-reducing ordering computed once per run (COLAMD, or METIS nested
// dissection through pymetis; orbit/core/solve.py:88-207,299-335).  The
// operator here is a 7-point stencil on a logically rectangular (nz, ny, nx)
// grid, so the ordering is computed geometrically: the box is cut recursively
// through its longest dimension by a one-cell-thick plane until a box holds at
// most `leaf_cells` cells.  Every plane (and every leaf box) is one supernode;
// its unknowns are eliminated after both half-boxes, and after elimination it
// is coupled densely to exactly the cells of ancestor planes that touch its box
// (the 6-neighbours of the box), which gives the multifrontal update sets
// without any graph search.  On a periodic-longitude grid a box that spans
// every column is a ring: cut across x it needs two planes (its first column
// and its middle column), which leave two ordinary boxes; the x-neighbours of
// a box touching column 0 or nx - 1 wrap around.
#include "symbolic.h"

#include <algorithm>
#include <cstdlib>
#include <array>
#include <cmath>
#include <functional>
#include <initializer_list>

namespace orbit {

namespace {

struct Box {
  int lo[3], hi[3];  // [k, j, i]
  int64_t cells() const {
    return int64_t(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
  }
};

struct Node {
  Box box;      // region of the subtree
  Box own;      // own cells (separator plane or the leaf box)
  Box own2;     // second separator plane of a ring cut across x (when two)
  bool two = false;
  bool ring = false;  // spans every column of a periodic grid
  int c[2] = {-1, -1};
  int parent = -1;
  int depth = 0;
};

}  // namespace

std::string build_symbolic(int nz, int ny, int nx, const SymbolicOptions& opt, Symbolic& S) {
  int leaf_cells = opt.leaf_cells;
  int chunk_elems = opt.chunk_elems;
  if (nz < 1 || ny < 1 || nx < 1) return "grid dimensions must be positive";
  if (opt.periodic_x && nx < 3) return "a periodic-longitude grid needs at least 3 columns";
  if (int64_t(nz) * ny * nx > (int64_t(1) << 30)) return "grid too large";
  if (leaf_cells < 1) leaf_cells = 1;
  if (chunk_elems < 256) chunk_elems = 256;
  S = Symbolic();
  S.nz = nz; S.ny = ny; S.nx = nx;
  S.periodic_x = opt.periodic_x ? 1 : 0;
  const bool px = S.periodic_x != 0;
  S.N = int64_t(nz) * ny * nx;
  S.leaf_cells = leaf_cells;
  const int64_t N = S.N;
  const int dims[3] = {nz, ny, nx};

  // ---- recursive dissection (explicit stack, postorder numbering) ----
  std::vector<Node> nodes;
  std::function<int(const Box&, int, int, bool)> rec = [&](const Box& b, int depth, int par, bool ring) -> int {
    Node nd;
    nd.box = b;
    nd.depth = depth;
    nd.parent = par;
    nd.ring = ring;
    int ext[3] = {b.hi[0] - b.lo[0], b.hi[1] - b.lo[1], b.hi[2] - b.lo[2]};
    int kids[2] = {-1, -1};
    if (b.cells() <= leaf_cells || (ext[0] <= 1 && ext[1] <= 1 && ext[2] <= 1)) {
      nd.own = b;
    } else {
      // longest dimension; ties prefer the horizontal axes (x, then y)
      int a = 2;
      if (ext[1] > ext[a]) a = 1;
      if (ext[0] > ext[a]) a = 0;
      int mid = (b.lo[a] + b.hi[a]) / 2;
      Box sep = b; sep.lo[a] = mid; sep.hi[a] = mid + 1;
      Box c1 = b; c1.hi[a] = mid;
      Box c2 = b; c2.lo[a] = mid + 1;
      bool kid_ring = ring;
      if (ring && a == 2) {
        // ring cut across x: planes at its first and middle columns
        Box sep0 = b; sep0.lo[2] = b.lo[2]; sep0.hi[2] = b.lo[2] + 1;
        nd.own = sep0;
        nd.own2 = sep;
        nd.two = true;
        c1.lo[2] = b.lo[2] + 1;
        kid_ring = false;
      } else {
        nd.own = sep;
      }
      int slot = 0;
      // children first (postorder), recorded after the recursion
      std::vector<Box> cb;
      if (c1.hi[a] > c1.lo[a]) cb.push_back(c1);
      if (c2.hi[a] > c2.lo[a]) cb.push_back(c2);
      for (auto& cbx : cb) kids[slot++] = rec(cbx, depth + 1, -2, kid_ring);
    }
    nd.c[0] = kids[0];
    nd.c[1] = kids[1];
    nodes.push_back(nd);
    int id = int(nodes.size()) - 1;
    for (int q = 0; q < 2; ++q)
      if (kids[q] >= 0) nodes[kids[q]].parent = id;
    return id;
  };
  Box root{{0, 0, 0}, {nz, ny, nx}};
  rec(root, 0, -1, px);
  const int ns = int(nodes.size());
  S.nsuper = ns;

  // ---- numbering ----
  S.perm.assign(N, -1);
  S.iperm.assign(N, -1);
  S.first.resize(ns); S.n.resize(ns); S.m.resize(ns); S.parent.resize(ns);
  S.level.resize(ns); S.nchild.resize(ns); S.child.assign(2 * ns, -1);
  int64_t next = 0;
  for (int s = 0; s < ns; ++s) {
    const Node& nd = nodes[s];
    S.first[s] = int32_t(next);
    for (int q = 0; q < (nd.two ? 2 : 1); ++q) {
      const Box& o = q ? nd.own2 : nd.own;
      for (int k = o.lo[0]; k < o.hi[0]; ++k)
        for (int j = o.lo[1]; j < o.hi[1]; ++j)
          for (int i = o.lo[2]; i < o.hi[2]; ++i) {
            int64_t cell = (int64_t(k) * ny + j) * nx + i;
            S.perm[next] = int32_t(cell);
            S.iperm[cell] = int32_t(next);
            ++next;
          }
    }
    S.n[s] = int32_t(next - S.first[s]);
    S.parent[s] = nd.parent;
    S.level[s] = nd.depth;
    S.nchild[s] = (nd.c[0] >= 0) + (nd.c[1] >= 0);
    S.child[2 * s] = nd.c[0];
    S.child[2 * s + 1] = nd.c[1];
  }
  if (next != N) return "internal: numbering does not cover the grid";
  S.sup_of.resize(N);
  for (int s = 0; s < ns; ++s)
    for (int q = 0; q < S.n[s]; ++q) S.sup_of[S.first[s] + q] = s;
  // first index of each subtree (postorder => contiguous range)
  std::vector<int32_t> sub_first(ns);
  for (int s = 0; s < ns; ++s) {
    int32_t f = S.first[s];
    for (int q = 0; q < 2; ++q)
      if (nodes[s].c[q] >= 0) f = std::min(f, sub_first[nodes[s].c[q]]);
    sub_first[s] = f;
  }

  // ---- update sets: 6-neighbours of the subtree box ----
  S.uoff.assign(ns + 1, 0);
  std::vector<std::vector<int32_t>> U(ns);
  for (int s = 0; s < ns; ++s) {
    const Box& b = nodes[s].box;
    std::vector<int32_t>& u = U[s];
    for (int a = 0; a < 3; ++a)
      for (int side = 0; side < 2; ++side) {
        if (a == 2 && nodes[s].ring) continue;  // a ring has no x-neighbours outside itself
        int plane = side == 0 ? b.lo[a] - 1 : b.hi[a];
        if (a == 2 && px) plane = (plane + nx) % nx;
        if (plane < 0 || plane >= dims[a]) continue;
        Box f = b;
        f.lo[a] = plane;
        f.hi[a] = plane + 1;
        for (int k = f.lo[0]; k < f.hi[0]; ++k)
          for (int j = f.lo[1]; j < f.hi[1]; ++j)
            for (int i = f.lo[2]; i < f.hi[2]; ++i) {
              int64_t cell = (int64_t(k) * ny + j) * nx + i;
              u.push_back(S.iperm[cell]);
            }
      }
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    int32_t last = S.first[s] + S.n[s];
    for (int32_t x : u)
      if (x < last) return "internal: update set reaches a non-ancestor";
    S.m[s] = int32_t(u.size());
    S.uoff[s + 1] = S.uoff[s] + int64_t(u.size());
  }
  S.uidx.resize(S.uoff[ns]);
  S.rel.resize(S.uoff[ns]);
  for (int s = 0; s < ns; ++s) {
    std::copy(U[s].begin(), U[s].end(), S.uidx.begin() + S.uoff[s]);
    int p = S.parent[s];
    for (size_t q = 0; q < U[s].size(); ++q) {
      int32_t x = U[s][q];
      int32_t pos = -1;
      if (p < 0) return "internal: root has a non-empty update set";
      if (x >= S.first[p] && x < S.first[p] + S.n[p]) {
        pos = x - S.first[p];
      } else {
        auto it = std::lower_bound(U[p].begin(), U[p].end(), x);
        if (it == U[p].end() || *it != x) return "internal: update set not inside the parent front";
        pos = S.n[p] + int32_t(it - U[p].begin());
      }
      S.rel[S.uoff[s] + q] = pos;
    }
  }
  // the solve's gathers rely on increasing extend-add maps (a parent's own
  // unknowns precede its ancestors in the elimination order)
  for (int s = 0; s < ns; ++s)
    for (int64_t q = S.uoff[s] + 1; q < S.uoff[s + 1]; ++q)
      if (S.rel[q] <= S.rel[q - 1]) return "internal: extend-add map not increasing";
  S.ginv_off.assign(ns + 1, 0);
  for (int s = 0; s < ns; ++s) S.ginv_off[s + 1] = S.ginv_off[s] + 2 * int64_t(S.n[s] + S.m[s]);
  S.ginv.assign(S.ginv_off[ns], -1);
  for (int s = 0; s < ns; ++s) {
    const int w = S.n[s] + S.m[s];
    for (int q = 0; q < 2; ++q) {
      const int c = S.child[2 * s + q];
      if (c < 0) continue;
      for (int u = 0; u < S.m[c]; ++u) S.ginv[S.ginv_off[s] + int64_t(q) * w + S.rel[S.uoff[c] + u]] = u;
    }
  }

  // ---- levels, storage ----
  int maxd = 0;
  for (int s = 0; s < ns; ++s) maxd = std::max(maxd, S.level[s]);
  S.nlevels = maxd + 1;
  S.level_sups.assign(S.nlevels, {});
  for (int s = 0; s < ns; ++s) S.level_sups[S.level[s]].push_back(s);
  S.ldn.resize(ns); S.ldm.resize(ns); S.ldf.resize(ns);
  S.fac_off.resize(ns); S.front_off.resize(ns); S.woff.resize(ns);
  S.level_front_size.assign(S.nlevels, 0);
  int64_t fo = 0, wo = 0;
  double flops = 0.0;
  for (int s = 0; s < ns; ++s) {
    int64_t n = S.n[s], m = S.m[s];
    S.ldn[s] = int32_t(round_up(n, kPad));
    S.ldm[s] = int32_t(round_up(std::max<int64_t>(m, 1), kPad));
    S.ldf[s] = int32_t(round_up(n + m, kPad));
    S.fac_off[s] = fo;
    fo += (n + m) * S.ldn[s] + n * S.ldm[s];
    S.fac_nnz += n * n + 2 * n * m;
    S.woff[s] = wo;
    wo += m;
    int l = S.level[s];
    S.front_off[s] = S.level_front_size[l];
    S.level_front_size[l] += (n + m) * S.ldf[s];
    S.max_front = std::max<int>(S.max_front, int(n + m));
    S.max_nm = std::max<int>(S.max_nm, int(std::max(n, m)));
    double nn = double(n), mm = double(m);
    flops += (2.0 / 3.0) * (std::pow(nn + mm, 3) - std::pow(mm, 3)) + (2.0 / 3.0) * nn * nn * nn +
             2.0 * mm * nn * nn;
  }
  S.factor_flops = flops;
  S.fac_size = fo;
  S.w_size = std::max<int64_t>(wo, 1);
  for (int l = 0; l < S.nlevels; ++l) S.front_buf_size = std::max(S.front_buf_size, S.level_front_size[l]);

  // ---- original-entry scatter lists (grouped by level) ----
  // Entry (row p, col q) of the permuted matrix lives in the front of the
  // supernode owning min(p, q).
  auto local_pos = [&](int s, int32_t x) -> int32_t {
    if (x >= S.first[s] && x < S.first[s] + S.n[s]) return x - S.first[s];
    const int32_t* b = S.uidx.data() + S.uoff[s];
    const int32_t* e = S.uidx.data() + S.uoff[s + 1];
    const int32_t* it = std::lower_bound(b, e, x);
    if (it == e || *it != x) return -1;
    return S.n[s] + int32_t(it - b);
  };
  std::vector<std::vector<std::pair<int64_t, int32_t>>> ent(S.nlevels);
  const int di[7] = {0, -1, 1, 0, 0, 0, 0};
  const int dj[7] = {0, 0, 0, -1, 1, 0, 0};
  const int dk[7] = {0, 0, 0, 0, 0, -1, 1};
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int64_t cell = (int64_t(k) * ny + j) * nx + i;
        for (int d = 0; d < 7; ++d) {
          int kk = k + dk[d], jj = j + dj[d], ii = i + di[d];
          if (px) ii = (ii + nx) % nx;
          if (kk < 0 || kk >= nz || jj < 0 || jj >= ny || ii < 0 || ii >= nx) continue;
          int64_t nb = (int64_t(kk) * ny + jj) * nx + ii;
          int32_t p = S.iperm[cell], q = S.iperm[nb];
          int s = S.sup_of[std::min(p, q)];
          int32_t lr = local_pos(s, p), lc = local_pos(s, q);
          if (lr < 0 || lc < 0) return "internal: matrix entry outside its front";
          ent[S.level[s]].push_back({S.front_off[s] + int64_t(lr) * S.ldf[s] + lc,
                                     int32_t(d * N + cell)});
        }
      }
  S.ent_level_off.assign(S.nlevels + 1, 0);
  for (int l = 0; l < S.nlevels; ++l) {
    std::sort(ent[l].begin(), ent[l].end());
    S.ent_level_off[l + 1] = S.ent_level_off[l] + int64_t(ent[l].size());
  }
  S.ent_pos.reserve(S.ent_level_off[S.nlevels]);
  S.ent_src.reserve(S.ent_level_off[S.nlevels]);
  for (int l = 0; l < S.nlevels; ++l)
    for (auto& pr : ent[l]) {
      S.ent_pos.push_back(pr.first);
      S.ent_src.push_back(pr.second);
    }

  // ---- factorization schedule ----
  S.tc_min_n = std::max(1, opt.tc_min_n);
  S.tc_pack_off.assign(ns, -1);
  S.tc_pack_size = 0;
  auto push_item = [&](int a, int b, int c, int d) {
    S.fitems.push_back(a); S.fitems.push_back(b); S.fitems.push_back(c); S.fitems.push_back(d);
  };
  auto nitems = [&]() { return int64_t(S.fitems.size() / 4); };
  S.fuse_max_n = std::max(0, std::min(kFrontMaxN, opt.fuse_max_n));
  S.n_fused = 0;
  for (int l = S.nlevels - 1; l >= 0; --l) {
    const auto& all = S.level_sups[l];
    // one-CTA fronts (FRONT) and the supernodes that take the blocked launches
    std::vector<int32_t> fused, sups;
    for (int s : all) {
      const bool one = S.m[s] > 0 && S.n[s] > 0 && S.n[s] <= S.fuse_max_n &&
                       front_smem_elems(S.n[s], S.m[s]) <= kFrontMaxElems;
      (one ? fused : sups).push_back(s);
    }
    S.n_fused += int64_t(fused.size());
    std::vector<int> small, big;  // tensor-core nodes: n >= tc_min_n and m > 0
    for (int s : sups) {
      if (S.m[s] == 0 || S.n[s] == 0) continue;
      (S.n[s] >= S.tc_min_n ? big : small).push_back(s);
    }
    {
      // every front row written once: the children's Schur complements
      // gathered through the inverse maps, zeros elsewhere; then the stencil
      // entries are added (SCATTER)
      int64_t off = nitems();
      for (int s : all) {
        const int w = S.n[s] + S.m[s];
        const int rows = 32;
        for (int r0 = 0; r0 < w; r0 += rows) push_item(s, r0, std::min(w, r0 + rows), 0);
      }
      S.fsched.push_back({FactorLaunch::ASSEMBLE, l, 0, off, nitems() - off});
    }
    S.fsched.push_back({FactorLaunch::SCATTER, l, 0, S.ent_level_off[l],
                        S.ent_level_off[l + 1] - S.ent_level_off[l]});
    {
      // one-CTA fronts in three shared-memory size classes, so that a launch
      // of small fronts is not held to the occupancy of the largest one
      const int64_t cls[3] = {4096, 12288, kFrontMaxElems};
      std::vector<char> done(fused.size(), 0);
      for (int c = 0; c < 3; ++c) {
        const int64_t off = nitems();
        int64_t emax = 0;
        for (size_t q = 0; q < fused.size(); ++q) {
          const int s = fused[q];
          const int64_t e = front_smem_elems(S.n[s], S.m[s]);
          if (done[q] || e > cls[c]) continue;
          done[q] = 1;
          emax = std::max(emax, e);
          push_item(s, 0, 0, 0);
        }
        if (nitems() > off) S.fsched.push_back({FactorLaunch::FRONT, l, int(emax), off, nitems() - off});
      }
    }
    int nmax = 0;
    for (int s : sups) nmax = std::max(nmax, S.n[s]);
    for (int p0 = 0; p0 < nmax; p0 += kNB) {
      int64_t off = nitems();
      for (int s : sups)
        if (S.n[s] > p0) push_item(s, 0, 0, 0);
      S.fsched.push_back({FactorLaunch::DIAG, l, p0, off, nitems() - off});
      off = nitems();
      for (int s : sups) {
        if (S.n[s] <= p0) continue;
        int nb = std::min(kNB, S.n[s] - p0);
        int rest = S.n[s] + S.m[s] - (p0 + nb);
        for (int ch = 0; ch * kTile < rest; ++ch) {
          push_item(s, 0, ch, 0);
          push_item(s, 1, ch, 0);
        }
      }
      if (nitems() > off) S.fsched.push_back({FactorLaunch::PANEL, l, p0, off, nitems() - off});
      off = nitems();
      for (int s : sups) {
        if (S.n[s] <= p0) continue;
        int nb = std::min(kNB, S.n[s] - p0);
        int rest = S.n[s] + S.m[s] - (p0 + nb);
        int nt = (rest + kSchurTile - 1) / kSchurTile;
        const int q0 = p0 + nb;
        // only 128-tiles touching the pivot rows or columns; the ancestor
        // block F22 is updated once, after the last pivot block (SCHUR)
        for (int tr = 0; tr < nt; ++tr)
          for (int tc = 0; tc < nt; ++tc)
            if (q0 + kSchurTile * tr < S.n[s] || q0 + kSchurTile * tc < S.n[s]) push_item(s, tr, tc, 0);
      }
      if (nitems() > off) S.fsched.push_back({FactorLaunch::UPDATE, l, p0, off, nitems() - off});
    }
    {
      // Schur complements on the CUDA cores: nodes below the tensor-core
      // threshold first (their item count goes in p0), then the tensor-core
      // nodes, which an fp32 factorization handles in its own pipeline below.
      int64_t off = nitems();
      int nsmall = 0;
      for (int pass = 0; pass < 2; ++pass)
        for (int s : pass == 0 ? small : big) {
          const int nt = (S.m[s] + kSchurTile - 1) / kSchurTile;
          for (int tr = 0; tr < nt; ++tr)
            for (int tc = 0; tc < nt; ++tc) push_item(s, tr, tc, 0);
          if (pass == 0) nsmall += nt * nt;
        }
      if (nitems() > off) S.fsched.push_back({FactorLaunch::SCHUR, l, nsmall, off, nitems() - off});
    }
    // blocked triangular inverses: step t fills block row t of Linv and block column t of Uinv
    int tmax = (nmax + kNB - 1) / kNB;
    for (int t = 1; t < tmax; ++t) {
      int64_t off = nitems();
      for (int s : sups) {
        int nbk = (S.n[s] + kNB - 1) / kNB;
        if (nbk <= t) continue;
        for (int j = 0; j < t; ++j) {
          push_item(s, 0, j, t);
          push_item(s, 1, j, t);
        }
      }
      if (nitems() > off) S.fsched.push_back({FactorLaunch::INV, l, t * kNB, off, nitems() - off});
    }
    // panel products via dense triangles copied into the pivot block
    for (int which = 0; which < 2; ++which) {
      int64_t off = nitems();
      for (int s : sups)
        if (S.m[s] > 0)
          for (int rb = 0; rb * 16 < S.n[s]; ++rb) push_item(s, rb, 0, 0);
      if (nitems() > off)
        S.fsched.push_back({which == 0 ? FactorLaunch::TRIL : FactorLaunch::TRIU, l, 0, off, nitems() - off});
      off = nitems();
      for (int s : sups) {
        const int tn = (S.n[s] + kSchurTile - 1) / kSchurTile, tm = (S.m[s] + kSchurTile - 1) / kSchurTile;
        if (S.m[s] == 0) continue;
        if (which == 0) {
          for (int a = 0; a < tm; ++a)
            for (int b = 0; b < tn; ++b) push_item(s, a, b, 0);  // Pb tile (rows of m, cols of n)
        } else {
          for (int a = 0; a < tn; ++a)
            for (int b = 0; b < tm; ++b) push_item(s, a, b, 0);  // Qr tile (rows of n, cols of m)
        }
      }
      if (nitems() > off)
        S.fsched.push_back({which == 0 ? FactorLaunch::PRODL : FactorLaunch::PRODU, l, 0, off, nitems() - off});
    }
    // Tensor-core pipeline of the fp32 factorization for the big nodes, whose
    // LU the panel/update launches above confined to F11 (F21, F12 stay as
    // assembled): X = inv(U11) inv(L11); Pb = -F21 X; Qr = -X F12; then the
    // Schur complement F22 += Pb F12.  Each GEMM reads operands packed as tf32
    // hi/lo tiles; pack items are {s, op, tile, k-block}, GEMM items
    // {s, row tile, column tile, job}.  Per node the pack holds F21 and F12^T
    // (mt x kt tiles each), inv(U11), inv(L11)^T, X and X^T (nt x kt each) and
    // Pb (mt x kt); the X GEMM writes the X packs and the Pb GEMM the Pb pack
    // from their epilogues.
    if (!big.empty()) {
      int64_t pack = 0;
      for (int s : big) {
        const int64_t mt = (S.m[s] + kSchurTile - 1) / kSchurTile, nt = (S.n[s] + kSchurTile - 1) / kSchurTile;
        const int64_t kt = (S.n[s] + kTcK - 1) / kTcK;
        S.tc_pack_off[s] = pack;
        pack += (3 * mt + 4 * nt) * kt * 2 * kTcTileFloats;
      }
      S.tc_pack_size = std::max(S.tc_pack_size, pack);
      auto pack_launch = [&](std::initializer_list<int> ops) {
        const int64_t off = nitems();
        for (int s : big) {
          const int mt = (S.m[s] + kSchurTile - 1) / kSchurTile, nt = (S.n[s] + kSchurTile - 1) / kSchurTile;
          const int kt = (S.n[s] + kTcK - 1) / kTcK;
          for (int op : ops) {
            const int tiles = (op == 0 || op == 1 || op == 6) ? mt : nt;
            for (int t = 0; t < tiles; ++t)
              for (int k = 0; k < kt; k += kTcPackRun) push_item(s, op, t, k);
          }
        }
        S.fsched.push_back({FactorLaunch::TC_PACK, l, 0, off, nitems() - off});
      };
      auto gemm_launch = [&](std::initializer_list<int> jobs) {
        const int64_t off = nitems();
        for (int s : big) {
          const int mt = (S.m[s] + kSchurTile - 1) / kSchurTile, nt = (S.n[s] + kSchurTile - 1) / kSchurTile;
          for (int job : jobs) {
            const int rows = (job == 0 || job == 2) ? nt : mt, cols = (job == 0 || job == 1) ? nt : mt;
            for (int a = 0; a < rows; ++a)
              for (int b = 0; b < cols; ++b) push_item(s, a, b, job);
          }
        }
        S.fsched.push_back({FactorLaunch::TC_GEMM, l, 0, off, nitems() - off});
      };
      pack_launch({0, 1, 2, 3});  // F21, F12^T, inv(U11), inv(L11)^T
      gemm_launch({0});           // X (and its packs)
      gemm_launch({1, 2});        // Pb (and its pack), Qr
      gemm_launch({3});           // Schur complement
    }
  }

  // ---- solve schedules ----
  // Rows of a supernode are split into chunks of roughly `chunk_elems`
  // matrix elements so that large separators spread over many CTAs.  Three
  // schedules (chunk/2, chunk, 2 chunk) serve small, medium and large
  // batches: fewer, larger chunks cost less per task when many orbits keep
  // the GPU busy, smaller ones shorten the critical path of a single orbit.
  // Subtree tasks: below a work threshold a whole subtree is one task (its
  // nodes are a contiguous postorder range), which removes the per-level
  // dependency waits of the many small supernodes near the leaves.
  std::vector<int64_t> subw(ns, 0);
  std::vector<int32_t> sub_node_first(ns);
  for (int s = 0; s < ns; ++s) {
    int64_t w = int64_t(S.n[s]) * S.n[s] + 2 * int64_t(S.n[s]) * S.m[s];
    int32_t f = s;
    for (int q = 0; q < 2; ++q) {
      int c = S.child[2 * s + q];
      if (c >= 0) {
        w += subw[c];
        f = std::min(f, sub_node_first[c]);
      }
    }
    subw[s] = w;
    sub_node_first[s] = f;
  }
  // Off by default: with several rows per warp in the chunked tasks, per-node
  // chunks beat whole-subtree tasks at every batch size measured (1 to 12
  // orbits).  subtree_div = d merges subtrees below fac_nnz / d work.
  const int64_t wmax = opt.subtree_div > 0 ? std::max<int64_t>(1, S.fac_nnz / opt.subtree_div) : 0;
  // role: 0 = chunked node, 1 = subtree root, 2 = inside a subtree
  S.role.assign(ns, 0);
  for (int s = ns - 1; s >= 0; --s) {
    const int p = S.parent[s];
    if (p >= 0 && S.role[p] != 0) S.role[s] = 2;
    else if (subw[s] <= wmax && (S.nchild[s] > 0 || p < 0 || subw[p] > wmax)) S.role[s] = 1;
  }
  S.max_sub_front = 0;
  for (int s2 = 0; s2 < ns; ++s2)
    if (S.role[s2] != 0) S.max_sub_front = std::max(S.max_sub_front, S.n[s2] + S.m[s2]);
  for (int k = 0; k < kNumSched; ++k) {
    SolveSched& Q = S.sched[k];
    Q.chunk_elems = k == 0 ? std::max(256, chunk_elems / 2) : k == 1 ? chunk_elems : 2 * chunk_elems;
    Q.nchunk_fwd.assign(ns, 0); Q.nchunk_bwd.assign(ns, 0);
    Q.nchunk_fwdT.assign(ns, 0); Q.nchunk_bwdT.assign(ns, 0);
    // Transposed sweeps (kinds 2, 3) work one column per lane: their chunks
    // hold at least 32 columns so that every lane of a warp has one.
    auto chunk_rows = [&](int s, int kind, int rows, std::function<int64_t(int)> rowlen) {
      int start = 0;
      int cnt = 0;
      int64_t acc = 0;
      const int min_rows = kind >= 2 ? 32 : 1;
      for (int r = 0; r < rows; ++r) {
        acc += std::max<int64_t>(rowlen(r), 1) + 8;
        bool last = (r == rows - 1);
        if ((acc >= Q.chunk_elems && r + 1 - start >= min_rows) || last || (r + 1 - start) >= 1024) {
          Q.sitems.push_back(s); Q.sitems.push_back(start); Q.sitems.push_back(r + 1);
          Q.sitems.push_back(kind);
          start = r + 1;
          acc = 0;
          ++cnt;
        }
      }
      return cnt;
    };
    auto push4 = [&](int a, int b, int c, int d) {
      Q.sitems.push_back(a); Q.sitems.push_back(b); Q.sitems.push_back(c); Q.sitems.push_back(d);
    };
    // non-transposed: fwd levels deep->0, bwd levels 0->deep
    Q.phase_off.clear();
    for (int l = S.nlevels - 1; l >= 0; --l) {
      Q.phase_off.push_back(int32_t(Q.sitems.size() / 4));
      for (int s : S.level_sups[l]) {
        int n = S.n[s], m = S.m[s];
        if (S.role[s] == 2) continue;
        if (S.role[s] == 1) {
          push4(s, sub_node_first[s], 0, 4);
          Q.nchunk_fwd[s] = 1;
          continue;
        }
        Q.nchunk_fwd[s] = chunk_rows(s, 0, n + m, [n](int r) { return r < n ? int64_t(r) : int64_t(n); });
      }
    }
    for (int l = 0; l < S.nlevels; ++l) {
      Q.phase_off.push_back(int32_t(Q.sitems.size() / 4));
      for (int s : S.level_sups[l]) {
        int n = S.n[s], m = S.m[s];
        if (S.role[s] == 2) continue;
        if (S.role[s] == 1) {
          push4(s, sub_node_first[s], 0, 5);
          Q.nchunk_bwd[s] = 1;
          continue;
        }
        Q.nchunk_bwd[s] = chunk_rows(s, 1, n, [n, m](int r) { return int64_t(n - r + m); });
      }
    }
    Q.phase_off.push_back(int32_t(Q.sitems.size() / 4));
    Q.items_per_bin = Q.phase_off.back();
    // transposed: fwdT levels deep->0 over output columns (n+m), bwdT levels 0->deep over n columns
    int32_t base = Q.items_per_bin;
    Q.phase_offT.clear();
    for (int l = S.nlevels - 1; l >= 0; --l) {
      Q.phase_offT.push_back(int32_t(Q.sitems.size() / 4) - base);
      for (int s : S.level_sups[l]) {
        int n = S.n[s], m = S.m[s];
        if (S.role[s] == 2) continue;
        if (S.role[s] == 1) {
          push4(s, sub_node_first[s], 0, 6);
          Q.nchunk_fwdT[s] = 1;
          continue;
        }
        Q.nchunk_fwdT[s] = chunk_rows(s, 2, n + m, [n](int c) { return c < n ? int64_t(c + 1) : int64_t(n); });
      }
    }
    for (int l = 0; l < S.nlevels; ++l) {
      Q.phase_offT.push_back(int32_t(Q.sitems.size() / 4) - base);
      for (int s : S.level_sups[l]) {
        int n = S.n[s], m = S.m[s];
        if (S.role[s] == 2) continue;
        if (S.role[s] == 1) {
          push4(s, sub_node_first[s], 0, 7);
          Q.nchunk_bwdT[s] = 1;
          continue;
        }
        Q.nchunk_bwdT[s] = chunk_rows(s, 3, n, [n, m](int c) { return int64_t(n - c + m); });
      }
    }
    Q.phase_offT.push_back(int32_t(Q.sitems.size() / 4) - base);
    Q.items_per_binT = Q.phase_offT.back();
  }
  return std::string();
}

}  // namespace orbit
