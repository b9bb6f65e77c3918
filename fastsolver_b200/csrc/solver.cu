// solver.cu -- device-resident HODLR system and its level schedule.
//
// The reference launches one Legion task per leaf and per (node, leaf) pair
// and lets region privileges order them (src/solver/fast_solver.cc:136-255).
// Here the same dependence structure is a fixed schedule on one stream:
//   1. every leaf at once: getrf + getrs (solver_tasks.cc:424-450);
//   2. for each depth d from the deepest internal level up to the root, every
//      internal node of depth d at once:
//        reduce  V_c^T [d_c | u_c] for both children (gemm.cc:208-229, as
//                split-K partial sums, summed in a fixed order by the node
//                kernel instead of REDOP_ADD atomics),
//        node    capacitance LU and eta (solver_tasks.cc:139-305),
//        bcast   d_c -= u_c eta (gemm.cc:232-284).
// Nodes of equal depth touch disjoint rows, so batching them does not change
// any operation's inputs; the leaf solves have no inputs from other tasks.
// All launch descriptors are built once per system and live on the device,
// so a solve is a fixed sequence of launches (capturable in a CUDA graph).
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>

#include "gemm_simt.cuh"
#include "leaf.cuh"
#include "leaf_blocked.cuh"
#include "node.cuh"
#include "solver.h"

namespace hodlr {

namespace {

template <typename T, typename TE>
struct PathSpec {
  T *X = nullptr;           // d columns (and the U columns on factor paths)
  long long ldx = 0;
  const T *Usrc = nullptr;  // transformed U columns (== X on factor paths)
  long long ldu = 0;
  T *D = nullptr;           // leaf LU factors
  long long ldd = 0;
  int *ipiv = nullptr, *perm = nullptr;
  const T *V = nullptr;
  long long ldv = 0;
  T *part = nullptr;   // split-K partial slots
  T *wfin = nullptr;   // summed W per child (when a child has several slots)
  TE *eta = nullptr;
  TE *M = nullptr;     // per-node solve matrices, (2r)^2 each
  NodeStore *ns = nullptr;
  const LeafPlan<T> *factors = nullptr;  // apply paths: the blocked leaf factors
  int nb_force = 0;                      // leaf panel width (0: by the largest leaf)
  int ob = 0;                            // leaf outer block width (0: one level)
  bool factor = false;
  int red_chunk = 512, bc_chunk = 512;
  int max_slots = 64;  // split-K slots per child at most
  int leaf_size = 1;  // nodes with at most this many real leaves use the 2r x 2r form
};

// Rows per split-K slot of a child with `nrow` rows: at least `chunk` rows,
// at most `max_slots` slots (the slots are summed into one W per child).
// The factor passes use up to 64 slots of >= 512 rows (wide products, few
// long tiles per SM); the FP32 refinement sweeps, whose products have only
// m columns, up to 1024 slots of >= 128 rows, so that the persistent sweep
// kernel's reduce step has many short units instead of a few long ones.
constexpr int kMaxSlots = 64;
constexpr int kSweepChunk = 128, kSweepMaxSlots = 1024;
inline int slot_rows(int nrow, int chunk, int max_slots = kMaxSlots) {
  const int ns = std::max(1, std::min(cdiv(nrow, chunk), max_slots));
  return cdiv(cdiv(nrow, ns), 16) * 16;
}

// Partial-sum, summed-W and eta workspace (elements) of a path's largest level.
void path_need(const Tree &t, bool factor, int chunk, size_t &part, size_t &wfin, size_t &eta,
               int max_slots = kMaxSlots) {
  part = wfin = eta = 0;
  for (int d = t.max_depth - 1; d >= 0; --d) {
    size_t p = 0, w = 0, e = 0;
    for (int id : t.internal_at_depth[d]) {
      const Node &P = t.nodes[id];
      const Node &c0 = t.nodes[P.lchild], &c1 = t.nodes[P.rchild];
      const int cw = factor ? c0.col_beg : t.nrhs;
      for (const Node *c : {&c0, &c1}) {
        const int NW = factor ? c->col_beg + c->ncol : t.nrhs;
        const int ns = cdiv(c->nrow, slot_rows(c->nrow, chunk, max_slots));
        p += (size_t)ns * c->vncol * NW;
        if (ns > 1) w += (size_t)c->vncol * NW;
      }
      e += (size_t)(c0.ncol + c1.ncol) * cw;
    }
    part = std::max(part, p);
    wfin = std::max(wfin, w);
    eta = std::max(eta, e);
  }
}


// Step lists of the two-level blocked leaf factorization (see LeafPlan and
// leaf_blocked.cu): forward steps on [D | X], then the backward solve on X.
// Every step is one merged launch over all leaves; a leaf without work in a
// step contributes no item.
template <typename T>
void build_leaf_plan(const Tree &t, T *Dbase, long long ldd, T *Xbase, long long ldx,
                     int *ipiv, int *perm, bool factor_cols_all, int m, LeafPlan<T> &lp,
                     int nb_force, int ob_req) {
  using Step = typename LeafPlan<T>::Step;
  const int nleaf = (int)t.leaves.size();
  lp.max_n = 0;
  for (int id : t.leaves) lp.max_n = std::max(lp.max_n, t.nodes[id].nrow);
  const int NB = nb_force > 0 ? nb_force : leaf_nb<T>(lp.max_n);
  const int OB = ob_req >= NB ? ob_req / NB * NB : NB;
  const int P = OB / NB;
  lp.nb = NB;
  lp.ob = OB;
  const int max_panels = cdiv(lp.max_n, NB);
  lp.nblocks = cdiv(lp.max_n, OB);
  lp.Linv.ensure((size_t)nleaf * max_panels * NB * NB);
  lp.Uinv.ensure((size_t)nleaf * max_panels * NB * NB);
  // block-row solves by the inverses of the outer diagonal blocks: in place
  // on the block's rows, which one GEMM tile row (128) covers (the GEMM
  // launchers run launches of items of at most 128 rows as 128-row tiles)
  const bool binv = P > 1 && OB <= 128;
  lp.binv = binv;
  if (binv) {
    lp.LinvB.ensure((size_t)nleaf * lp.nblocks * OB * OB);
    lp.UinvB.ensure((size_t)nleaf * lp.nblocks * OB * OB);
  }
  lp.swapflag.ensure((size_t)nleaf * max_panels);
  std::vector<LeafFactorTask<T>> tasks(nleaf);
  lp.laswp_cols = 0;
  for (int q = 0; q < nleaf; ++q) {
    const Node &nd = t.nodes[t.leaves[q]];
    LeafFactorTask<T> &k = tasks[q];
    k.D = Dbase + nd.row_beg;
    k.ldd = ldd;
    k.X = Xbase + nd.row_beg;
    k.ldx = ldx;
    k.ipiv = ipiv + nd.row_beg;
    k.perm = perm + nd.row_beg;
    k.Linv = lp.Linv.p + (size_t)q * max_panels * NB * NB;
    k.Uinv = lp.Uinv.p + (size_t)q * max_panels * NB * NB;
    k.swapflag = lp.swapflag.p + (size_t)q * max_panels;
    k.LinvB = binv ? lp.LinvB.p + (size_t)q * lp.nblocks * OB * OB : nullptr;
    k.UinvB = binv ? lp.UinvB.p + (size_t)q * lp.nblocks * OB * OB : nullptr;
    k.n = nd.nrow;
    k.ncols = factor_cols_all ? nd.col_beg + nd.ncol : m;
    k.info_slot = q;
    lp.laswp_cols = std::max(lp.laswp_cols, k.n + k.ncols);
  }
  lp.tasks.upload(tasks);
  lp.host_tasks = tasks;
  lp.nleaf = nleaf;
  lp.fwd.clear();
  lp.bwd.clear();
  // item lists of one GEMM step, filled leaf by leaf
  struct Acc {
    std::vector<GemmItem<T, T>> it;
    std::vector<GemmSeg<T>> sg;
    void add(T *C, long long ldc, int M, int N, const T *A, long long lda, const T *B,
             long long ldb, int K, bool inplace) {
      if (M <= 0 || N <= 0 || K <= 0) return;
      GemmSeg<T> g{A, B, lda, ldb, K, 0};
      GemmItem<T, T> i{C, inplace ? C : nullptr, ldc, inplace ? ldc : 0, M, N, (int)sg.size(), 1};
      sg.push_back(g);
      it.push_back(i);
    }
  };
  auto gemm_step = [&](typename LeafPlan<T>::Kind kind, const Acc &a) {
    auto st = std::make_unique<Step>();
    st->kind = kind;
    st->g.set(a.it, a.sg);
    return st;
  };
  auto laswp_step = [&](int p0, int np, int a0, int a1, int b0, int b1, bool with_x) {
    auto st = std::make_unique<Step>();
    st->kind = LeafPlan<T>::kLaswp;
    st->panel = p0;
    st->np = np;
    st->a0 = a0; st->a1 = a1; st->b0 = b0; st->b1 = b1;
    st->with_x = with_x;
    return st;
  };
  constexpr int kAll = 1 << 30;
  for (int J = 0; J < lp.nblocks; ++J) {
    const int j0 = J * OB;
    // the block's panels: factor, interchange and update inside the block columns
    for (int p = 0; p < P; ++p) {
      const int pi = J * P + p, k0 = pi * NB;
      auto pan = std::make_unique<Step>();
      pan->kind = LeafPlan<T>::kPanel;
      pan->k0 = k0;
      pan->panel = pi;
      lp.fwd.push_back(std::move(pan));
      lp.fwd.push_back(laswp_step(pi, 1, j0, k0, k0 + NB, j0 + OB, false));
      Acc tr, up;
      for (const LeafFactorTask<T> &k : tasks) {
        if (k0 >= k.n) continue;
        const int kb = std::min(NB, k.n - k0);
        const int N = std::min(j0 + OB, k.n) - (k0 + kb);
        const int rest = k.n - k0 - kb;
        const T *Li = k.Linv + (size_t)pi * NB * NB;
        T *U12 = k.D + k0 + (long long)(k0 + kb) * ldd;
        tr.add(U12, ldd, kb, N, Li, NB, U12, ldd, kb, false);
        up.add(k.D + (k0 + kb) + (long long)(k0 + kb) * ldd, ldd, rest, N,
               k.D + (k0 + kb) + (long long)k0 * ldd, ldd, U12, ldd, kb, true);
      }
      lp.fwd.push_back(gemm_step(LeafPlan<T>::kTrsm, tr));
      lp.fwd.push_back(gemm_step(LeafPlan<T>::kUpdate, up));
    }
    // the block's interchanges on the columns left and right of it and on X
    lp.fwd.push_back(laswp_step(J * P, P, 0, j0, j0 + OB, kAll, true));
    if (binv) {
      // block rows: U12 = L11^{-1} A12 on R = (D right of the block | X), one
      // product with the inverse of the block's unit-lower triangle
      auto inv = std::make_unique<Step>();
      inv->kind = LeafPlan<T>::kBlockInv;
      inv->block = J;
      lp.fwd.push_back(std::move(inv));
      Acc tr;
      for (const LeafFactorTask<T> &k : tasks) {
        if (j0 >= k.n) continue;
        const int obe = std::min(OB, k.n - j0);
        const T *Li = k.LinvB + (size_t)J * OB * OB;
        T *Dr = k.D + j0 + (long long)(j0 + obe) * ldd;
        T *Xr = k.X + j0;
        tr.add(Dr, ldd, obe, k.n - j0 - obe, Li, OB, Dr, ldd, obe, false);
        tr.add(Xr, ldx, obe, k.ncols, Li, OB, Xr, ldx, obe, false);
      }
      lp.fwd.push_back(gemm_step(LeafPlan<T>::kTrsm, tr));
    }
    // block rows: U12 = L11^{-1} A12 by panels on R = (D right of the block | X)
    for (int p = 0; p < (binv ? 0 : P); ++p) {
      const int pi = J * P + p, k0 = pi * NB;
      Acc tr, up;
      for (const LeafFactorTask<T> &k : tasks) {
        if (k0 >= k.n) continue;
        const int kb = std::min(NB, k.n - k0);
        const int obe = std::min(OB, k.n - j0);
        const int nd = k.n - j0 - obe;           // D columns right of the block
        const int below = j0 + obe - k0 - kb;    // block rows below this panel
        const T *Li = k.Linv + (size_t)pi * NB * NB;
        T *Dr = k.D + k0 + (long long)(j0 + obe) * ldd;
        T *Xr = k.X + k0;
        tr.add(Dr, ldd, kb, nd, Li, NB, Dr, ldd, kb, false);
        tr.add(Xr, ldx, kb, k.ncols, Li, NB, Xr, ldx, kb, false);
        const T *L = k.D + (k0 + kb) + (long long)k0 * ldd;
        up.add(Dr + kb, ldd, below, nd, L, ldd, Dr, ldd, kb, true);
        up.add(Xr + kb, ldx, below, k.ncols, L, ldd, Xr, ldx, kb, true);
      }
      lp.fwd.push_back(gemm_step(LeafPlan<T>::kTrsm, tr));
      lp.fwd.push_back(gemm_step(LeafPlan<T>::kUpdate, up));
    }
    // trailing update of depth OB: A22 -= L21 U12 on R, rows below the block
    Acc big;
    for (const LeafFactorTask<T> &k : tasks) {
      if (j0 >= k.n) continue;
      const int obe = std::min(OB, k.n - j0);
      const int rest = k.n - j0 - obe;
      const T *L21 = k.D + (j0 + obe) + (long long)j0 * ldd;
      big.add(k.D + (j0 + obe) + (long long)(j0 + obe) * ldd, ldd, rest, rest, L21, ldd,
              k.D + j0 + (long long)(j0 + obe) * ldd, ldd, obe, true);
      big.add(k.X + (j0 + obe), ldx, rest, k.ncols, L21, ldd, k.X + j0, ldx, obe, true);
    }
    lp.fwd.push_back(gemm_step(LeafPlan<T>::kUpdate, big));
  }
  lp.fwd_per_block = binv ? 4 * P + 4 : 6 * P + 2;
  // backward solve on X, last block first
  for (int J = lp.nblocks - 1; J >= 0; --J) {
    const int j0 = J * OB;
    if (binv) {
      // X[block] = U11^{-1} X[block]: one product with the block's upper inverse
      Acc tr;
      for (const LeafFactorTask<T> &k : tasks) {
        if (j0 >= k.n) continue;
        const int obe = std::min(OB, k.n - j0);
        T *Xk = k.X + j0;
        tr.add(Xk, ldx, obe, k.ncols, k.UinvB + (size_t)J * OB * OB, OB, Xk, ldx, obe, false);
      }
      lp.bwd.push_back(gemm_step(LeafPlan<T>::kTrsm, tr));
    }
    for (int p = binv ? -1 : P - 1; p >= 0; --p) {
      const int pi = J * P + p, k0 = pi * NB;
      Acc tr, up;
      for (const LeafFactorTask<T> &k : tasks) {
        if (k0 >= k.n) continue;
        const int kb = std::min(NB, k.n - k0);
        T *Xk = k.X + k0;
        tr.add(Xk, ldx, kb, k.ncols, k.Uinv + (size_t)pi * NB * NB, NB, Xk, ldx, kb, false);
        up.add(k.X + j0, ldx, k0 - j0, k.ncols, k.D + j0 + (long long)k0 * ldd, ldd, Xk, ldx,
               kb, true);
      }
      lp.bwd.push_back(gemm_step(LeafPlan<T>::kTrsm, tr));
      lp.bwd.push_back(gemm_step(LeafPlan<T>::kUpdate, up));
    }
    Acc big;
    for (const LeafFactorTask<T> &k : tasks) {
      if (j0 >= k.n) continue;
      const int obe = std::min(OB, k.n - j0);
      big.add(k.X, ldx, j0, k.ncols, k.D + (long long)j0 * ldd, ldd, k.X + j0, ldx, obe, true);
    }
    lp.bwd.push_back(gemm_step(LeafPlan<T>::kUpdate, big));
  }
  lp.bwd_per_block = binv ? 2 : 2 * P + 1;
}

template <typename TA, typename TC, typename TACC>
void run_gemm(const GemmLaunch<TA, TC> &g, bool trans, TACC alpha, TACC beta, cudaStream_t s) {
  launch_gemm_items<TA, TC, TACC>(g.items.p, g.segs.p, g.n, g.max_m, g.max_n, trans, alpha, beta,
                                  s);
}

template <typename T>
void run_leaf_plan(Profiler &pf, const LeafPlan<T> &lp, int *info, cudaStream_t s);

// The level descriptors of an FP32 apply path for the persistent sweep
// kernel, when every level's products have at most 32 columns.
template <typename T, typename TE>
void build_sweep(PathPlan<T, TE> &plan) {
  plan.sweep_ok = false;
  if constexpr (std::is_same<T, float>::value && std::is_same<TE, float>::value) {
    if (plan.factor || plan.levels.empty()) return;
    std::vector<SweepLevel> v;
    int mx = 0;
    for (const auto &Lp : plan.levels) {
      const LevelPlan<T, TE> &L = *Lp;
      if (L.red_max_n > 32 || L.ap_max_n > 32 || L.bc_max_n > 32) return;
      SweepLevel d{};
      d.red_items = L.red_items.p;
      d.red_segs = L.red_segs.p;
      d.n_red = L.n_red;
      d.red_mt = cdiv(std::max(L.red_max_m, 1), 64);
      d.red_nt = cdiv(std::max(L.red_max_n, 1), 16);
      d.sums = L.sums.p;
      d.n_sums = L.n_sums;
      d.sum_units = (int)cdiv<long long>(std::max<long long>(L.sum_max_len, 1), kSweepSumChunk);
      d.sum_max_slots = L.sum_max_slots;
      d.ap_items = L.ap_items.p;
      d.ap_segs = L.ap_segs.p;
      d.n_ap = L.n_ap;
      d.ap_rb = cdiv(std::max(L.ap_max_m, 1), 128);
      d.bc_items = L.bc_items.p;
      d.bc_segs = L.bc_segs.p;
      d.n_bc = L.n_bc;
      d.bc_rb = cdiv(std::max(L.bc_max_m, 1), 128);
      mx = std::max(mx, std::max(L.ap_max_n, L.bc_max_n));
      v.push_back(d);
    }
    plan.sweep.upload(v);
    plan.sweep_bar.ensure(kSweepBarWords);
    plan.sweep_max_n = std::max(mx, 1);
    plan.sweep_ok = true;
  }
}

template <typename T, typename TE>
void build_path(const Tree &t, const PathSpec<T, TE> &sp, PathPlan<T, TE> &plan, int form) {
  plan.levels.clear();
  plan.factor = sp.factor;
  const int m = t.nrhs;
  std::vector<LeafTask<T>> lt;
  plan.max_n = plan.max_nrhs = 0;
  for (size_t q = 0; q < t.leaves.size(); ++q) {
    const Node &n = t.nodes[t.leaves[q]];
    LeafTask<T> k{};
    k.D = sp.D + n.row_beg;
    k.ldd = sp.ldd;
    k.X = sp.X + n.row_beg;
    k.ldx = sp.ldx;
    k.ipiv = sp.ipiv + n.row_beg;
    k.perm = sp.perm + n.row_beg;
    k.n = n.nrow;
    k.nrhs = sp.factor ? n.col_beg + n.ncol : m;
    k.info_slot = (int)q;
    plan.max_n = std::max(plan.max_n, k.n);
    plan.max_nrhs = std::max(plan.max_nrhs, k.nrhs);
    lt.push_back(k);
  }
  plan.nleaf = (int)lt.size();
  plan.leaf_tasks.upload(lt);
  if (sp.factor) {
    build_leaf_plan<T>(t, sp.D, sp.ldd, sp.X, sp.ldx, sp.ipiv, sp.perm, true, m, plan.leaf,
                       sp.nb_force, sp.ob);
  } else if (sp.factors) {
    std::vector<LeafFactorTask<T>> at = sp.factors->host_tasks;
    for (size_t q = 0; q < at.size(); ++q) {
      const Node &n = t.nodes[t.leaves[q]];
      at[q].X = sp.X + n.row_beg;
      at[q].ldx = sp.ldx;
      at[q].ncols = m;
    }
    plan.apply_tasks.upload(at);
    plan.apply_nb = sp.factors->nb;
    plan.apply_max_n = sp.factors->max_n;
    plan.apply_max_cols = m;
  }
  const int nleaf = (int)t.leaves.size();

  for (int d = t.max_depth - 1; d >= 0; --d) {
    const auto &ids = t.internal_at_depth[d];
    if (ids.empty()) continue;
    auto L = std::make_unique<LevelPlan<T, TE>>();
    std::vector<GemmItem<T, T>> ri, bi;
    std::vector<GemmSeg<T>> rs, bs;
    std::vector<NodeTask<T, TE>> nt[2];
    std::vector<SumTask<T>> su;
    std::vector<GemmItem<T, double>> gi;
    std::vector<GemmSeg<T>> gs;
    std::vector<GemmItem<T, T>> ai;
    std::vector<GemmSeg<T>> as;
    size_t poff = 0, woff = 0, eoff = 0;
    L->v_lo = 1 << 30;
    for (int p : ids) {
      const Node &P = t.nodes[p];
      const Node &c0 = t.nodes[P.lchild], &c1 = t.nodes[P.rchild];
      const int cw = sp.factor ? c0.col_beg : m;
      for (const Node *c : {&c0, &c1}) {
        L->v_lo = std::min(L->v_lo, c->col_beg - m);
        L->v_hi = std::max(L->v_hi, c->col_beg - m + c->vncol);
      }
      NodeTask<T, TE> k{};
      const T *W0d = nullptr, *W1d = nullptr;
      long long ldw0d = 0, ldw1d = 0;
      for (int side = 0; side < 2; ++side) {
        const Node &c = side ? c1 : c0;
        const int NW = sp.factor ? c.col_beg + c.ncol : m;
        const int M = c.vncol;
        const int rows_per = slot_rows(c.nrow, sp.red_chunk, sp.max_slots);
        const int nslots = cdiv(c.nrow, rows_per);
        T *slot0 = sp.part + poff;
        for (int q = 0; q < nslots; ++q) {
          const int rb = c.row_beg + q * rows_per;
          const int rows = std::min(rows_per, c.row_beg + c.nrow - rb);
          GemmSeg<T> sg{};
          sg.A = sp.V + rb + (long long)(c.col_beg - m) * sp.ldv;
          sg.B = sp.X + rb;
          sg.lda = sp.ldv;
          sg.ldb = sp.ldx;
          sg.K = rows;
          GemmItem<T, T> it{};
          it.C = slot0 + (size_t)q * M * NW;
          it.Cin = nullptr;
          it.ldc = M;
          it.M = M;
          it.N = NW;
          it.seg_begin = (int)rs.size();
          it.seg_count = 1;
          rs.push_back(sg);
          ri.push_back(it);
          L->red_max_m = std::max(L->red_max_m, M);
          L->red_max_n = std::max(L->red_max_n, NW);
        }
        poff += (size_t)nslots * M * NW;
        T *W = slot0;
        if (nslots > 1) {
          W = sp.wfin + woff;
          woff += (size_t)M * NW;
          SumTask<T> st{};
          st.dst = W;
          st.src = slot0;
          st.len = (long long)M * NW;
          st.stride = (long long)M * NW;
          st.nslots = nslots;
          su.push_back(st);
          L->sum_max_len = std::max(L->sum_max_len, st.len);
          L->sum_max_slots = std::max(L->sum_max_slots, nslots);
        }
        if (side == 0) {
          W0d = W; k.W0u = W + (size_t)M * (NW - c.ncol);
          ldw0d = k.ldw0u = M;
        } else {
          W1d = W; k.W1u = W + (size_t)M * (NW - c.ncol);
          ldw1d = k.ldw1u = M;
        }
      }
      const int r0 = c0.ncol, r1 = c1.ncol, s2 = r0 + r1;
      k.r0 = r0;
      k.r1 = r1;
      // eta = [eta0; eta1] (s2 x cw, ld s2): eta0 feeds child 0, eta1 child 1
      TE *eta = sp.eta + eoff;
      eoff += (size_t)s2 * cw;
      k.S = sp.ns->S.p + (size_t)p * sp.ns->rr;
      k.F = sp.ns->F.p + (size_t)p * sp.ns->rr;
      k.M = sp.M + (size_t)p * sp.ns->mm;
      k.info_slot = nleaf + p;
      // the node's form: 1 everywhere when asked for, else 1 inside a Legion leaf
      const int nform = (form == 1 || inside_legion_leaf(t, p, sp.leaf_size)) ? 1 : 0;
      nt[nform].push_back(k);
      if (sp.factor && nform == 0) {
        // S = I - V1Tu1 V0Tu0 (r0 x r0, ld r0): the dgemm at solver_tasks.cc:261
        GemmSeg<T> g{};
        g.A = k.W1u;
        g.lda = k.ldw1u;
        g.B = k.W0u;
        g.ldb = k.ldw0u;
        g.K = r1;
        GemmItem<T, double> it{};
        it.C = sp.ns->S.p + (size_t)p * sp.ns->rr;
        it.ldc = r0;
        it.Cin = sp.ns->ident.p;
        it.ldcin = t.rank;
        it.M = it.N = r0;
        it.seg_begin = (int)gs.size();
        it.seg_count = 1;
        gs.push_back(g);
        gi.push_back(it);
        L->gram_max = std::max(L->gram_max, r0);
      }
      const int s = nform == 0 ? r0 : s2;
      L->max_s[nform] = std::max(L->max_s[nform], s);
      L->max_r[nform] = std::max(L->max_r[nform], std::max(r0, r1));
      if (cw > 0) {
        // [eta0; eta1] = M [V0Td0; V1Td1]: one item, two K segments
        GemmSeg<T> a0{}, a1{};
        a0.A = reinterpret_cast<const T *>(k.M);
        a0.lda = s2;
        a0.B = W0d;
        a0.ldb = ldw0d;
        a0.K = r1;
        a1.A = reinterpret_cast<const T *>(k.M) + (size_t)r1 * s2;
        a1.lda = s2;
        a1.B = W1d;
        a1.ldb = ldw1d;
        a1.K = r0;
        GemmItem<T, T> it{};
        it.C = reinterpret_cast<T *>(eta);
        it.ldc = s2;
        it.M = s2;
        it.N = cw;
        it.seg_begin = (int)as.size();
        it.seg_count = 2;
        as.push_back(a0);
        as.push_back(a1);
        ai.push_back(it);
        L->ap_max_m = std::max(L->ap_max_m, s2);
        L->ap_max_n = std::max(L->ap_max_n, cw);
      }
      // broadcast d_c -= u_c eta into both children
      for (int side = 0; side < 2; ++side) {
        const Node &c = side ? c1 : c0;
        const TE *eta_c = side ? eta + r0 : eta;
        if (cw == 0) continue;
        for (int rb = c.row_beg; rb < c.row_beg + c.nrow; rb += sp.bc_chunk) {
          const int rows = std::min(sp.bc_chunk, c.row_beg + c.nrow - rb);
          GemmSeg<T> sg{};
          sg.A = sp.Usrc + rb + (long long)c.col_beg * sp.ldu;
          sg.B = reinterpret_cast<const T *>(eta_c);
          sg.lda = sp.ldu;
          sg.ldb = s2;
          sg.K = c.ncol;
          GemmItem<T, T> it{};
          it.C = sp.X + rb;
          it.Cin = sp.X + rb;
          it.ldc = it.ldcin = sp.ldx;
          it.M = rows;
          it.N = cw;
          it.seg_begin = (int)bs.size();
          it.seg_count = 1;
          bs.push_back(sg);
          bi.push_back(it);
          L->bc_max_m = std::max(L->bc_max_m, rows);
          L->bc_max_n = std::max(L->bc_max_n, cw);
        }
      }
    }
    L->red_items.upload(ri);
    L->red_segs.upload(rs);
    L->n_red = (int)ri.size();
    L->sums.upload(su);
    L->n_sums = (int)su.size();
    L->gram_items.upload(gi);
    L->gram_segs.upload(gs);
    L->n_gram = (int)gi.size();
    for (int f = 0; f < 2; ++f) {
      L->node_tasks[f].upload(nt[f]);
      L->n_nodes[f] = (int)nt[f].size();
      L->g_alias[f] = node_g_alias(nt[f]);
    }
    L->ap_items.upload(ai);
    L->ap_segs.upload(as);
    L->n_ap = (int)ai.size();
    L->bc_items.upload(bi);
    L->bc_segs.upload(bs);
    L->n_bc = (int)bi.size();
    plan.levels.push_back(std::move(L));
  }
  build_sweep(plan);
  plan.built = true;
}

// RAII phase marker: records a CUDA event pair when profiling is on.
struct PhaseScope {
  Profiler &p;
  int ph;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  PhaseScope(Profiler &p_, int ph_, cudaStream_t s_) : p(p_), ph(ph_), s(s_) {
    if (p.on) p.begin(ph, s, a);
  }
  ~PhaseScope() {
    if (p.on) p.end(ph, s, a);
  }
};

template <typename T>
void run_leaf_plan(Profiler &pf, const LeafPlan<T> &lp, int *info, cudaStream_t s) {
  using Step = typename LeafPlan<T>::Step;
  auto run_step = [&](const Step &st) {
    switch (st.kind) {
      case LeafPlan<T>::kPanel: {
        PhaseScope pp(pf, PH_LEAF_PANEL, s);
        launch_leaf_panel<T>(lp.tasks.p, lp.nleaf, lp.max_n, lp.nb, st.k0, st.panel, info, s);
        break;
      }
      case LeafPlan<T>::kLaswp: {
        if (st.a1 <= st.a0 && st.b1 <= st.b0 && !st.with_x) break;  // no columns
        PhaseScope pp(pf, PH_LEAF_PANEL, s);
        launch_leaf_laswp<T>(lp.tasks.p, lp.nleaf, lp.laswp_cols, lp.nb, st.panel, st.np, st.a0,
                             st.a1, st.b0, st.b1, st.with_x, s);
        break;
      }
      case LeafPlan<T>::kBlockInv: {
        PhaseScope pt(pf, PH_LEAF_TRSM, s);
        launch_leaf_block_inverse<T>(lp.tasks.p, lp.nleaf, lp.nb, lp.ob, st.block, false, 0, s);
        break;
      }
      case LeafPlan<T>::kTrsm: {
        if (st.g.n == 0) break;
        PhaseScope pt(pf, PH_LEAF_TRSM, s);
        run_gemm<T, T, T>(st.g, false, T(1), T(0), s);
        break;
      }
      case LeafPlan<T>::kUpdate: {
        if (st.g.n == 0) break;
        PhaseScope pu(pf, PH_LEAF_UPDATE, s);
        run_gemm<T, T, T>(st.g, false, T(-1), T(1), s);
        break;
      }
    }
  };
  {
    PhaseScope ps(pf, PH_GETRF, s);
    launch_leaf_init<T>(lp.tasks.p, lp.nleaf, info, s);
    for (const auto &st : lp.fwd) run_step(*st);
    if (lp.binv) {  // the upper block inverses of every block, for the backward solve
      PhaseScope pt(pf, PH_LEAF_TRSM, s);
      launch_leaf_block_inverse<T>(lp.tasks.p, lp.nleaf, lp.nb, lp.ob, 0, true, lp.nblocks, s);
    }
  }
  {
    PhaseScope ps(pf, PH_GETRS, s);
    for (const auto &st : lp.bwd)
      if (st->g.n > 0)
        run_gemm<T, T, T>(st->g, false, st->kind == LeafPlan<T>::kTrsm ? T(1) : T(-1),
                          st->kind == LeafPlan<T>::kTrsm ? T(0) : T(1), s);
  }
}

// parts: kPathLeaves (the leaf solves / factorization), kPathLevels (the
// tree levels), or both; the levels read nothing of V before their first
// reduce, so a caller can let V arrive in between
template <typename T, typename TE>
void run_path(Profiler &pf, const PathPlan<T, TE> &plan, int form, int *info, cudaStream_t s,
              int parts = kPathLeaves | kPathLevels, const LevelHook *hook = nullptr) {
  LeafTask<T> none{};
  if (!(parts & kPathLeaves)) {
  } else if (plan.factor) {
    run_leaf_plan<T>(pf, plan.leaf, info, s);
  } else if (plan.apply_nb > 0) {
    PhaseScope ps(pf, PH_GETRS, s);
    launch_leaf_apply<T>(plan.apply_tasks.p, plan.nleaf, plan.apply_max_n, plan.apply_max_cols,
                         plan.apply_nb, s);
  } else {
    PhaseScope ps(pf, PH_GETRS, s);
    launch_getrs<T>(plan.leaf_tasks.p, none, plan.nleaf, plan.max_n, plan.max_nrhs, s);
  }
  if (!(parts & kPathLevels)) return;
  if (!plan.factor && plan.sweep_ok && sweep_persistent_enabled()) {
    PhaseScope ps(pf, PH_SWEEP_LEVELS, s);
    launch_sweep_levels(plan.sweep.p, (int)plan.levels.size(), plan.sweep_max_n,
                        plan.sweep_bar.p, s);
    return;
  }
  int li = 0;
  for (const auto &Lp : plan.levels) {
    const LevelPlan<T, TE> &L = *Lp;
    if (hook) (*hook)(li, L.v_lo, L.v_hi);
    ++li;
    {
      PhaseScope ps(pf, PH_REDUCE, s);
      launch_gemm_items<T, T, T>(L.red_items.p, L.red_segs.p, L.n_red, L.red_max_m,
                                 L.red_max_n, true, T(1), T(0), s);
      launch_sum_slots<T>(L.sums.p, L.n_sums, L.sum_max_len, s);
    }
    if (plan.factor) {
      PhaseScope ps(pf, PH_NODE_FACTOR, s);
      // S = I - V1Tu1 V0Tu0 for the form-0 nodes, unless the node kernel stages
      // its inputs and forms S itself
      if (L.n_gram > 0 && !(L.n_nodes[0] > 0 && node_factor_stages(L.max_s[0], L.max_r[0])))
        launch_gemm_items<T, double, double>(L.gram_items.p, L.gram_segs.p, L.n_gram, L.gram_max,
                                             L.gram_max, false, -1.0, 1.0, s);
      for (int f = 0; f < 2; ++f)
        if (L.n_nodes[f] > 0)
          launch_node_factor<T, TE>(L.node_tasks[f].p, L.n_nodes[f], L.max_s[f], L.max_r[f], f,
                                    info, s, L.g_alias[f]);
    }
    {
      PhaseScope ps(pf, PH_NODE_APPLY, s);
      launch_gemm_items<T, T, T>(L.ap_items.p, L.ap_segs.p, L.n_ap, L.ap_max_m, L.ap_max_n,
                                 false, T(1), T(0), s);
    }
    {
      PhaseScope ps(pf, PH_BCAST, s);
      launch_gemm_items<T, T, T>(L.bc_items.p, L.bc_segs.p, L.n_bc, L.bc_max_m, L.bc_max_n,
                                 false, T(-1), T(1), s);
    }
  }
}

void alloc_node_store(NodeStore &ns, const Tree &t, bool fp64) {
  const int r = t.rank;
  ns.rr = r * r;
  ns.mm = 4 * r * r;
  const size_t nn = t.nodes.size();
  ns.S.ensure(nn * ns.rr);
  ns.F.ensure(nn * ns.rr);
  if (fp64) ns.M64.ensure(nn * ns.mm);
  else ns.M32.ensure(nn * ns.mm);
  std::vector<double> I((size_t)r * r, 0.0);
  for (int i = 0; i < r; ++i) I[(size_t)i * r + i] = 1.0;
  ns.ident.upload(I);
}

void build_matvec(System &S, const double *x, MatvecPlan &mv) {
  const Tree &t = S.tree;
  const int m = S.m;
  const long long N = S.N;
  const int chunk = 1024;
  std::vector<GemmItem<double, double>> ri, ai;
  std::vector<GemmSeg<double>> rs, as;
  std::vector<SumTask<double>> su;
  std::vector<size_t> toff(t.nodes.size(), 0);
  size_t poff = 0, tsz = 0;
  for (size_t i = 1; i < t.nodes.size(); ++i) {
    const Node &c = t.nodes[i];
    toff[i] = tsz;
    tsz += (size_t)c.vncol * m;
  }
  size_t pneed = 0;
  for (size_t i = 1; i < t.nodes.size(); ++i) {
    const int rp = slot_rows(t.nodes[i].nrow, chunk);
    pneed += (size_t)cdiv(t.nodes[i].nrow, rp) * t.nodes[i].vncol * m;
  }
  S.tbuf.ensure(std::max<size_t>(tsz, 1));
  S.mvpart.ensure(std::max<size_t>(pneed, 1));
  mv.red_max_m = mv.red_max_n = 0;
  for (size_t i = 1; i < t.nodes.size(); ++i) {
    const Node &c = t.nodes[i];
    const int M = c.vncol;
    const int rows_per = slot_rows(c.nrow, chunk);
    const int nslots = cdiv(c.nrow, rows_per);
    double *slot0 = S.mvpart.p + poff;
    for (int q = 0; q < nslots; ++q) {
      const int rb = c.row_beg + q * rows_per;
      const int rows = std::min(rows_per, c.row_beg + c.nrow - rb);
      GemmSeg<double> sg{};
      sg.A = S.V.p + rb + (long long)(c.col_beg - m) * N;
      sg.B = x + rb;
      sg.lda = N;
      sg.ldb = N;
      sg.K = rows;
      GemmItem<double, double> it{};
      it.C = slot0 + (size_t)q * M * m;
      it.ldc = M;
      it.M = M;
      it.N = m;
      it.seg_begin = (int)rs.size();
      it.seg_count = 1;
      rs.push_back(sg);
      ri.push_back(it);
      mv.red_max_m = std::max(mv.red_max_m, M);
      mv.red_max_n = std::max(mv.red_max_n, m);
    }
    SumTask<double> st{};
    st.dst = S.tbuf.p + toff[i];
    st.src = slot0;
    st.len = (long long)M * m;
    st.stride = (long long)M * m;
    st.nslots = nslots;
    su.push_back(st);
    mv.sum_max_len = std::max(mv.sum_max_len, st.len);
    poff += (size_t)nslots * M * m;
  }
  mv.ap_max_m = mv.ap_max_n = 0;
  for (int leaf : t.leaves) {
    const Node &n = t.nodes[leaf];
    GemmItem<double, double> it{};
    it.C = S.R64.p + n.row_beg;
    it.Cin = S.B.p + n.row_beg;
    it.ldc = N;
    it.ldcin = N;
    it.M = n.nrow;
    it.N = m;
    it.seg_begin = (int)as.size();
    GemmSeg<double> sd{};
    sd.A = S.D.p + n.row_beg;
    sd.lda = N;
    sd.B = x + n.row_beg;
    sd.ldb = N;
    sd.K = n.nrow;
    as.push_back(sd);
    for (int a = leaf; a > 0; a = t.nodes[a].parent) {
      const Node &an = t.nodes[a];
      const Node &pa = t.nodes[an.parent];
      const int sib = (pa.lchild == a) ? pa.rchild : pa.lchild;
      GemmSeg<double> su_{};
      su_.A = S.U.p + n.row_beg + (long long)(an.col_beg - m) * N;
      su_.lda = N;
      su_.B = S.tbuf.p + toff[sib];
      su_.ldb = an.ncol;
      su_.K = an.ncol;
      as.push_back(su_);
    }
    it.seg_count = (int)as.size() - it.seg_begin;
    ai.push_back(it);
    mv.ap_max_m = std::max(mv.ap_max_m, n.nrow);
    mv.ap_max_n = std::max(mv.ap_max_n, m);
  }
  mv.red_items.upload(ri);
  mv.red_segs.upload(rs);
  mv.n_red = (int)ri.size();
  mv.sums.upload(su);
  mv.n_sums = (int)su.size();
  mv.ap_items.upload(ai);
  mv.ap_segs.upload(as);
  mv.n_ap = (int)ai.size();
  mv.built = true;
}

// ---- merging the plans of several systems into one batch schedule.  All
// descriptors hold absolute device pointers into their own system's buffers,
// so merging is concatenation: item lists shift their segment indices, INFO
// slots shift by the system's offset in the batch's INFO array.

template <typename TA, typename TC>
struct ItemAcc {
  std::vector<GemmItem<TA, TC>> it;
  std::vector<GemmSeg<TA>> sg;
  int max_m = 0, max_n = 0;
  void add(const std::vector<GemmItem<TA, TC>> &items, const std::vector<GemmSeg<TA>> &segs) {
    const int off = (int)sg.size();
    for (GemmItem<TA, TC> x : items) {
      x.seg_begin += off;
      it.push_back(x);
      max_m = std::max(max_m, x.M);
      max_n = std::max(max_n, x.N);
    }
    sg.insert(sg.end(), segs.begin(), segs.end());
  }
  void add(const GemmLaunch<TA, TC> &g) { add(g.items.h, g.segs.h); }
  void store(GemmLaunch<TA, TC> &g) const { g.set(it, sg); }
  void store(DevBuf<GemmItem<TA, TC>> &items, DevBuf<GemmSeg<TA>> &segs, int &n, int &mm,
             int &mn) const {
    items.upload(it);
    segs.upload(sg);
    n = (int)it.size();
    mm = max_m;
    mn = max_n;
  }
};

template <typename T>
void merge_leaf_plans(const std::vector<const LeafPlan<T> *> &src, const std::vector<int> &info_off,
                      LeafPlan<T> &dst) {
  using Step = typename LeafPlan<T>::Step;
  std::vector<LeafFactorTask<T>> tasks;
  dst.max_n = dst.laswp_cols = 0;
  dst.nb = src.empty() ? 0 : src[0]->nb;
  dst.ob = src.empty() ? 0 : src[0]->ob;
  dst.nblocks = 0;
  for (size_t k = 0; k < src.size(); ++k) {
    const LeafPlan<T> &lp = *src[k];
    if (lp.nb != dst.nb || lp.ob != dst.ob) throw CudaError{cudaErrorInvalidValue};
    for (LeafFactorTask<T> t : lp.host_tasks) {
      t.info_slot += info_off[k];
      tasks.push_back(t);
    }
    dst.max_n = std::max(dst.max_n, lp.max_n);
    dst.laswp_cols = std::max(dst.laswp_cols, lp.laswp_cols);
    dst.nblocks = std::max(dst.nblocks, lp.nblocks);
  }
  dst.fwd_per_block = src[0]->fwd_per_block;
  dst.bwd_per_block = src[0]->bwd_per_block;
  dst.binv = src[0]->binv;
  dst.tasks.upload(tasks);
  dst.host_tasks = tasks;
  dst.nleaf = (int)tasks.size();
  dst.fwd.clear();
  dst.bwd.clear();
  // the step lists have the same shape per block in every system (same nb
  // and ob): step i of block J merges the systems that have block J; the
  // backward lists start at each system's own last block
  auto merge_step = [&](const Step &proto, const std::vector<const Step *> &parts) {
    auto st = std::make_unique<Step>();
    st->kind = proto.kind;
    st->k0 = proto.k0;
    st->panel = proto.panel;
    st->block = proto.block;
    st->np = proto.np;
    st->a0 = proto.a0; st->a1 = proto.a1; st->b0 = proto.b0; st->b1 = proto.b1;
    st->with_x = proto.with_x;
    if (proto.kind == LeafPlan<T>::kTrsm || proto.kind == LeafPlan<T>::kUpdate) {
      ItemAcc<T, T> acc;
      for (const Step *p : parts) acc.add(p->g);
      acc.store(st->g);
    }
    return st;
  };
  for (int J = 0; J < dst.nblocks; ++J)
    for (int i = 0; i < dst.fwd_per_block; ++i) {
      std::vector<const Step *> parts;
      for (const LeafPlan<T> *lp : src)
        if (J < lp->nblocks) parts.push_back(lp->fwd[(size_t)J * dst.fwd_per_block + i].get());
      dst.fwd.push_back(merge_step(*parts[0], parts));
    }
  for (int J = dst.nblocks - 1; J >= 0; --J)
    for (int i = 0; i < dst.bwd_per_block; ++i) {
      std::vector<const Step *> parts;
      for (const LeafPlan<T> *lp : src)
        if (J < lp->nblocks)
          parts.push_back(lp->bwd[(size_t)(lp->nblocks - 1 - J) * dst.bwd_per_block + i].get());
      dst.bwd.push_back(merge_step(*parts[0], parts));
    }
}

// Level j of the merged plan is level j (deepest first) of every system
// that has one: each system still walks its own levels bottom-up.
template <typename T, typename TE>
void merge_paths(const std::vector<const PathPlan<T, TE> *> &src, const std::vector<int> &info_off,
                 PathPlan<T, TE> &dst) {
  dst.levels.clear();
  dst.factor = src[0]->factor;
  dst.nleaf = 0;
  dst.max_n = dst.max_nrhs = 0;
  dst.apply_nb = dst.apply_max_n = dst.apply_max_cols = 0;
  if (dst.factor) {
    std::vector<const LeafPlan<T> *> lps;
    for (const auto *p : src) lps.push_back(&p->leaf);
    merge_leaf_plans<T>(lps, info_off, dst.leaf);
    dst.nleaf = dst.leaf.nleaf;
  } else {
    std::vector<LeafFactorTask<T>> at;
    for (const auto *p : src) {
      at.insert(at.end(), p->apply_tasks.h.begin(), p->apply_tasks.h.end());
      if (p->apply_nb != src[0]->apply_nb) throw CudaError{cudaErrorInvalidValue};
      dst.apply_max_n = std::max(dst.apply_max_n, p->apply_max_n);
      dst.apply_max_cols = std::max(dst.apply_max_cols, p->apply_max_cols);
    }
    dst.apply_tasks.upload(at);
    dst.apply_nb = src[0]->apply_nb;
    dst.nleaf = (int)at.size();
  }
  size_t nlev = 0;
  for (const auto *p : src) nlev = std::max(nlev, p->levels.size());
  for (size_t j = 0; j < nlev; ++j) {
    auto L = std::make_unique<LevelPlan<T, TE>>();
    ItemAcc<T, T> red, ap, bc;
    ItemAcc<T, double> gram;
    std::vector<SumTask<T>> su;
    std::vector<NodeTask<T, TE>> nt[2];
    for (size_t k = 0; k < src.size(); ++k) {
      if (j >= src[k]->levels.size()) continue;
      const LevelPlan<T, TE> &S = *src[k]->levels[j];
      red.add(S.red_items.h, S.red_segs.h);
      gram.add(S.gram_items.h, S.gram_segs.h);
      ap.add(S.ap_items.h, S.ap_segs.h);
      bc.add(S.bc_items.h, S.bc_segs.h);
      su.insert(su.end(), S.sums.h.begin(), S.sums.h.end());
      L->sum_max_len = std::max(L->sum_max_len, S.sum_max_len);
      L->sum_max_slots = std::max(L->sum_max_slots, S.sum_max_slots);
      for (int f = 0; f < 2; ++f) {
        for (NodeTask<T, TE> t : S.node_tasks[f].h) {
          t.info_slot += info_off[k];
          nt[f].push_back(t);
        }
        L->max_s[f] = std::max(L->max_s[f], S.max_s[f]);
        L->max_r[f] = std::max(L->max_r[f], S.max_r[f]);
      }
    }
    red.store(L->red_items, L->red_segs, L->n_red, L->red_max_m, L->red_max_n);
    int gm = 0, gn = 0;
    gram.store(L->gram_items, L->gram_segs, L->n_gram, gm, gn);
    L->gram_max = std::max(gm, gn);
    ap.store(L->ap_items, L->ap_segs, L->n_ap, L->ap_max_m, L->ap_max_n);
    bc.store(L->bc_items, L->bc_segs, L->n_bc, L->bc_max_m, L->bc_max_n);
    L->sums.upload(su);
    L->n_sums = (int)su.size();
    for (int f = 0; f < 2; ++f) {
      L->node_tasks[f].upload(nt[f]);
      L->n_nodes[f] = (int)nt[f].size();
      L->g_alias[f] = node_g_alias(nt[f]);
    }
    dst.levels.push_back(std::move(L));
  }
  build_sweep(dst);
  dst.built = true;
}

void merge_matvecs(const std::vector<const MatvecPlan *> &src, MatvecPlan &dst) {
  ItemAcc<double, double> red, ap;
  std::vector<SumTask<double>> su;
  dst.sum_max_len = 0;
  for (const MatvecPlan *p : src) {
    red.add(p->red_items.h, p->red_segs.h);
    ap.add(p->ap_items.h, p->ap_segs.h);
    su.insert(su.end(), p->sums.h.begin(), p->sums.h.end());
    dst.sum_max_len = std::max(dst.sum_max_len, p->sum_max_len);
  }
  red.store(dst.red_items, dst.red_segs, dst.n_red, dst.red_max_m, dst.red_max_n);
  ap.store(dst.ap_items, dst.ap_segs, dst.n_ap, dst.ap_max_m, dst.ap_max_n);
  dst.sums.upload(su);
  dst.n_sums = (int)su.size();
  dst.built = true;
}

void matvec_launches(Profiler &pf, const MatvecPlan &p, double alpha, double beta,
                     cudaStream_t s) {
  PhaseScope ps(pf, PH_MATVEC, s);
  launch_gemm_items<double, double, double>(p.red_items.p, p.red_segs.p, p.n_red, p.red_max_m,
                                            p.red_max_n, true, 1.0, 0.0, s);
  launch_sum_slots<double>(p.sums.p, p.n_sums, p.sum_max_len, s);
  launch_gemm_items<double, double, double>(p.ap_items.p, p.ap_segs.p, p.n_ap, p.ap_max_m,
                                            p.ap_max_n, false, alpha, beta, s);
}

}  // namespace

void Profiler::begin(int ph, cudaStream_t s, cudaEvent_t &a) {
  HODLR_CUDA_TRY(cudaEventCreate(&a));
  HODLR_CUDA_TRY(cudaEventRecord(a, s));
  (void)ph;
}
void Profiler::end(int ph, cudaStream_t s, cudaEvent_t a) {
  cudaEvent_t b;
  HODLR_CUDA_TRY(cudaEventCreate(&b));
  HODLR_CUDA_TRY(cudaEventRecord(b, s));
  recs.push_back({ph, a, b});
}
void Profiler::collect() {
  for (auto &r : recs) {
    HODLR_CUDA_TRY(cudaEventSynchronize(r.b));
    float t = 0.f;
    HODLR_CUDA_TRY(cudaEventElapsedTime(&t, r.a, r.b));
    ms[r.phase] += t;
    launches[r.phase] += 1;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  recs.clear();
}
void Profiler::reset() {
  collect();
  for (int i = 0; i < PH_COUNT; ++i) { ms[i] = 0; launches[i] = 0; }
}

int System::init(int N_, int nrhs, int rank, int threshold) {
  int rc = build_tree(N_, nrhs, rank, threshold, tree);
  if (rc) return rc;
  if (2 * rank > kMaxNodeS && rank > kMaxNodeS) return -3;
  N = N_;
  m = nrhs;
  r = rank;
  C = tree.ncols;
  vc = tree.vcols();
  nmax = tree.max_leaf;
  const size_t n = (size_t)N;
  D.ensure(n * nmax);
  U.ensure(n * std::max(vc, 1));
  V.ensure(n * std::max(vc, 1));
  B.ensure(n * m);
  Xsol.ensure(n * m);
  R64.ensure(n * m);
  MVx.ensure(n * m);
  relres_dev.ensure(m);
  ratio_part.ensure((size_t)m * kRatioChunks * 2);
  n_info = (int)(tree.leaves.size() + tree.nodes.size());
  info.ensure(n_info);
  HODLR_CUDA_TRY(cudaMemset(info.p, 0, sizeof(int) * n_info));
  HODLR_CUDA_TRY(cudaMemset(D.p, 0, sizeof(double) * n * nmax));
  HODLR_CUDA_TRY(cudaMemset(U.p, 0, sizeof(double) * n * std::max(vc, 1)));
  HODLR_CUDA_TRY(cudaMemset(V.p, 0, sizeof(double) * n * std::max(vc, 1)));
  HODLR_CUDA_TRY(cudaMemset(B.p, 0, sizeof(double) * n * m));
  HODLR_CUDA_TRY(cudaMemset(Xsol.p, 0, sizeof(double) * n * m));
  build_matvec(*this, Xsol.p, mv_sol);
  build_matvec(*this, MVx.p, mv_usr);
  return 0;
}

void System::ensure_fp64() {
  if (fused64[0].built) return;
  const size_t n = (size_t)N;
  X64.ensure(n * C);
  DLU64.ensure(n * nmax);
  Y64.ensure(n * m);
  ipiv64.ensure(n);
  perm64.ensure(n);
  alloc_node_store(ns64, tree, true);
  size_t pf, wf, ef, pa, wa, ea;
  path_need(tree, true, red_chunk, pf, wf, ef);
  path_need(tree, false, red_chunk, pa, wa, ea);
  part64.ensure(std::max<size_t>(std::max(pf, pa), 1));
  wfin64.ensure(std::max<size_t>(std::max(wf, wa), 1));
  eta64.ensure(std::max<size_t>(std::max(ef, ea), 1));
  for (int form = 0; form < 2; ++form) {
    if (form == 1 && 2 * r > kMaxNodeS) continue;
    PathSpec<double, double> f;
    f.X = X64.p; f.ldx = N; f.Usrc = X64.p; f.ldu = N;
    f.D = DLU64.p; f.ldd = N; f.ipiv = ipiv64.p; f.perm = perm64.p;
    f.V = V.p; f.ldv = N; f.part = part64.p; f.wfin = wfin64.p; f.eta = eta64.p; f.M = ns64.M64.p; f.ns = &ns64;
    f.factor = true; f.red_chunk = red_chunk; f.bc_chunk = bc_chunk; f.ob = ob64;
    f.leaf_size = leaf_size;
    build_path(tree, f, fused64[form], form);
    PathSpec<double, double> a = f;
    a.X = Y64.p; a.factor = false; a.factors = &fused64[form].leaf;
    build_path(tree, a, apply64[form], form);
  }
}

void System::ensure_mixed() {
  if (fused32.built) return;
  const size_t n = (size_t)N;
  X32.ensure(n * C);
  D32.ensure(n * nmax);
  V32.ensure(n * std::max(vc, 1));
  Y32.ensure(n * m);
  ipiv32.ensure(n);
  perm32.ensure(n);
  alloc_node_store(ns32, tree, false);
  size_t pf, wf, ef, pa, wa, ea;
  path_need(tree, true, red_chunk, pf, wf, ef);
  path_need(tree, false, kSweepChunk, pa, wa, ea, kSweepMaxSlots);
  part32.ensure(std::max<size_t>(std::max(pf, pa), 1));
  wfin32.ensure(std::max<size_t>(std::max(wf, wa), 1));
  eta32.ensure(std::max<size_t>(std::max(ef, ea), 1));
  PathSpec<float, float> f;
  f.X = X32.p; f.ldx = N; f.Usrc = X32.p; f.ldu = N;
  f.D = D32.p; f.ldd = N; f.ipiv = ipiv32.p; f.perm = perm32.p;
  f.V = V32.p; f.ldv = N; f.part = part32.p; f.wfin = wfin32.p; f.eta = eta32.p; f.M = ns32.M32.p; f.ns = &ns32;
  f.factor = true; f.red_chunk = red_chunk; f.bc_chunk = bc_chunk; f.nb_force = nb32;
  f.ob = ob32;
  build_path(tree, f, fused32, 0);
  PathSpec<float, float> a = f;
  a.X = Y32.p; a.factor = false; a.factors = &fused32.leaf;
  a.red_chunk = kSweepChunk;
  a.max_slots = kSweepMaxSlots;
  build_path(tree, a, apply32, 0);
}

void System::run_fused64(int form, cudaStream_t s) {
  ensure_fp64();
  const size_t n = (size_t)N;
  HODLR_CUDA_TRY(cudaMemcpyAsync(DLU64.p, D.p, sizeof(double) * n * nmax, cudaMemcpyDeviceToDevice, s));
  HODLR_CUDA_TRY(cudaMemcpyAsync(X64.p, B.p, sizeof(double) * n * m, cudaMemcpyDeviceToDevice, s));
  if (vc > 0)
    HODLR_CUDA_TRY(cudaMemcpyAsync(X64.p + n * m, U.p, sizeof(double) * n * vc,
                                   cudaMemcpyDeviceToDevice, s));
  run_path(prof, fused64[form], form, info.p, s);
  HODLR_CUDA_TRY(cudaMemcpyAsync(Xsol.p, X64.p, sizeof(double) * n * m, cudaMemcpyDeviceToDevice, s));
  factored = HODLR_PREC_FP64;
  factored_form = form;
}

void System::run_apply64(cudaStream_t s) {
  run_path(prof, apply64[factored_form], factored_form, nullptr, s);
}

void System::run_factor32(cudaStream_t s) {
  run_factor32_part(kPathLeaves | kPathLevels, s);
}

void System::run_factor32_part(int parts, cudaStream_t s) {
  convert32(parts, s);
  run_path(prof, fused32, 0, info.p, s, parts);
  if (parts & kPathLevels) {
    factored = HODLR_PREC_MIXED;
    factored_form = 0;
  }
}

void System::run_factor32_levels_hooked(const LevelHook &hook, cudaStream_t s) {
  ensure_mixed();
  run_path(prof, fused32, 0, info.p, s, kPathLevels, &hook);
  factored = HODLR_PREC_MIXED;
  factored_form = 0;
}

void System::convert_v32(int lo, int hi, cudaStream_t s) {
  if (hi <= lo) return;
  PhaseScope ps(prof, PH_CONVERT, s);
  launch_convert2d<double, float>(V.p + (size_t)lo * N, N, V32.p + (size_t)lo * N, N, N, hi - lo, s);
}

void System::convert32(int parts, cudaStream_t s) {
  ensure_mixed();
  const long long n = N;
  {
    PhaseScope ps(prof, PH_CONVERT, s);
    if (parts & kPathLeaves) {  // what the leaf factorization reads: D and [b | U]
      launch_convert2d<double, float>(D.p, n, D32.p, n, n, nmax, s);
      launch_convert2d<double, float>(B.p, n, X32.p, n, n, m, s);
      if (vc > 0) launch_convert2d<double, float>(U.p, n, X32.p + (size_t)n * m, n, n, vc, s);
    }
    if ((parts & kPathLevels) && vc > 0)  // V, first read by the levels' reduce
      launch_convert2d<double, float>(V.p, n, V32.p, n, n, vc, s);
  }
}

void System::run_apply32(cudaStream_t s) { run_path(prof, apply32, 0, nullptr, s); }

void System::run_matvec(const MatvecPlan &p, double alpha, double beta, cudaStream_t s) {
  matvec_launches(prof, p, alpha, beta, s);
}

int System::check_info(cudaStream_t s) {
  std::vector<int> h(n_info);
  HODLR_CUDA_TRY(cudaMemcpyAsync(h.data(), info.p, sizeof(int) * n_info, cudaMemcpyDeviceToHost, s));
  HODLR_CUDA_TRY(cudaStreamSynchronize(s));
  const int nleaf = (int)tree.leaves.size();
  for (int i = 0; i < n_info; ++i)
    if (h[i] != 0) return i < nleaf ? h[i] : 100000 + h[i];
  return 0;
}

void System::relres_enqueue(cudaStream_t s) {
  run_matvec(mv_sol, -1.0, 1.0, s);
  launch_colratio(R64.p, N, B.p, N, N, m, ratio_part.p, relres_dev.p, s);
}

double System::relres(cudaStream_t s) {
  relres_enqueue(s);
  return relres_read(s);
}

double System::relres_read(cudaStream_t s) {
  std::vector<double> h(m);
  HODLR_CUDA_TRY(cudaMemcpyAsync(h.data(), relres_dev.p, sizeof(double) * m,
                                 cudaMemcpyDeviceToHost, s));
  HODLR_CUDA_TRY(cudaStreamSynchronize(s));
  double mx = 0.0;
  for (double v : h) mx = std::max(mx, std::isnan(v) ? INFINITY : v);
  return mx;
}

// ---- Batch

void Batch::build(const std::vector<System *> &systems) {
  if (systems.empty()) throw CudaError{cudaErrorInvalidValue};
  sys = systems;
  groups.clear();
  for (size_t k = 0; k < sys.size(); ++k) {
    System *S = sys[k];
    S->ensure_mixed();
    const int nbk = S->fused32.leaf.nb, obk = S->fused32.leaf.ob;
    const bool wide = S->m > 16;
    Group *g = nullptr;
    for (auto &q : groups)
      if (q->nb == nbk && q->ob == obk && q->wide == wide) g = q.get();
    if (!g) {
      groups.push_back(std::make_unique<Group>());
      g = groups.back().get();
      g->nb = nbk;
      g->ob = obk;
      g->wide = wide;
    }
    g->members.push_back((int)k);
  }
  info_off.clear();
  rr_off.clear();
  n_info = 0;
  int n_rr = 0;
  max_m = 0;
  std::vector<const MatvecPlan *> mp;
  std::vector<Ew2DTask<double, float>> cin, cres;
  std::vector<Ew2DTask<float, double>> cx0, addy;
  std::vector<RatioTask> rt;
  for (System *S : sys) {
    info_off.push_back(n_info);
    n_info += S->n_info;
    rr_off.push_back(n_rr);
    n_rr += S->m;
    max_m = std::max(max_m, S->m);
    mp.push_back(&S->mv_sol);
    const long long n = S->N;
    auto add_in = [&](const double *src, float *dst, long long cols) {
      if (cols > 0) cin.push_back({src, n, dst, n, n, cols, 0});
    };
    add_in(S->D.p, S->D32.p, S->nmax);
    add_in(S->B.p, S->X32.p, S->m);
    add_in(S->U.p, S->X32.p + (size_t)n * S->m, S->vc);
    add_in(S->V.p, S->V32.p, S->vc);
    cres.push_back({S->R64.p, n, S->Y32.p, n, n, S->m, 0});
    cx0.push_back({S->X32.p, n, S->Xsol.p, n, n, S->m, 0});
    addy.push_back({S->Y32.p, n, S->Xsol.p, n, n, S->m, 0});
  }
  t_in = ew2d_prefix(cin);
  t_res = ew2d_prefix(cres);
  t_x0 = ew2d_prefix(cx0);
  ew2d_prefix(addy);
  rr.ensure(std::max(n_rr, 1));
  for (size_t k = 0; k < sys.size(); ++k) {
    System *S = sys[k];
    RatioTask t{};
    t.r = S->R64.p;
    t.ldr = S->N;
    t.b = S->B.p;
    t.ldb = S->N;
    t.rows = S->N;
    t.out = rr.p + rr_off[k];
    t.cols = S->m;
    rt.push_back(t);
  }
  for (auto &g : groups) {
    std::vector<const PathPlan<float, float> *> fp, ap;
    std::vector<int> off;
    for (int k : g->members) {
      fp.push_back(&sys[k]->fused32);
      ap.push_back(&sys[k]->apply32);
      off.push_back(info_off[k]);
    }
    merge_paths<float, float>(fp, off, g->fused32);
    merge_paths<float, float>(ap, off, g->apply32);
  }
  merge_matvecs(mp, mv);
  cv_in.upload(cin);
  cv_res.upload(cres);
  cv_x0.upload(cx0);
  add_y.upload(addy);
  ratios.upload(rt);
  info.ensure(n_info);
  HODLR_CUDA_TRY(cudaMemset(info.p, 0, sizeof(int) * n_info));
  g_factor.reset();
  g_sweep.reset();
}

void Batch::residuals(cudaStream_t s) {
  matvec_launches(prof, mv, -1.0, 1.0, s);
  launch_colratio_batched(ratios.p, (int)sys.size(), max_m, s);
}

void Batch::run_factor(cudaStream_t s) {
  {
    PhaseScope ps(prof, PH_CONVERT, s);
    launch_ew2d_batched<double, float>(cv_in.p, (int)cv_in.h.size(), t_in, false, s);
  }
  for (auto &g : groups) run_path(prof, g->fused32, 0, info.p, s);
  launch_ew2d_batched<float, double>(cv_x0.p, (int)cv_x0.h.size(), t_x0, false, s);
  residuals(s);
}

void Batch::run_sweep(cudaStream_t s) {
  launch_ew2d_batched<double, float>(cv_res.p, (int)cv_res.h.size(), t_res, false, s);
  for (auto &g : groups) run_path(prof, g->apply32, 0, nullptr, s);
  launch_ew2d_batched<float, double>(add_y.p, (int)add_y.h.size(), t_x0, true, s);
  residuals(s);
}

int Batch::check_info(cudaStream_t s, int *failed) {
  std::vector<int> h(n_info);
  HODLR_CUDA_TRY(cudaMemcpyAsync(h.data(), info.p, sizeof(int) * n_info, cudaMemcpyDeviceToHost, s));
  HODLR_CUDA_TRY(cudaStreamSynchronize(s));
  if (failed) *failed = -1;
  for (size_t k = 0; k < sys.size(); ++k) {
    const int nl = (int)sys[k]->tree.leaves.size();
    for (int i = 0; i < sys[k]->n_info; ++i) {
      const int v = h[info_off[k] + i];
      if (v == 0) continue;
      if (failed) *failed = (int)k;
      return i < nl ? v : 100000 + v;
    }
  }
  return 0;
}

double Batch::relres_read(cudaStream_t s, std::vector<double> *per_system) {
  const int n_rr = rr_off.back() + sys.back()->m;
  std::vector<double> h(n_rr);
  HODLR_CUDA_TRY(cudaMemcpyAsync(h.data(), rr.p, sizeof(double) * n_rr, cudaMemcpyDeviceToHost, s));
  HODLR_CUDA_TRY(cudaStreamSynchronize(s));
  double mx = 0.0;
  if (per_system) per_system->assign(sys.size(), 0.0);
  for (size_t k = 0; k < sys.size(); ++k) {
    double mk = 0.0;
    for (int c = 0; c < sys[k]->m; ++c) {
      const double v = h[rr_off[k] + c];
      mk = std::max(mk, std::isnan(v) ? INFINITY : v);
    }
    if (per_system) (*per_system)[k] = mk;
    mx = std::max(mx, mk);
  }
  return mx;
}

}  // namespace hodlr
