// solver.h -- one HODLR system on the device and the level schedule that
// replaces fastSolver's Legion task launches (FastSolver::bfs_solve,
// src/solver/fast_solver.cc:56-72, 136-255).
#pragma once

#include <functional>
#include <memory>
#include <vector>

#include "common.cuh"
#include "htree.h"
#include "leaf_blocked.cuh"
#include "sweep.cuh"
#include "util.cuh"

namespace hodlr {

// Grow-only device buffer.
template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  std::vector<T> h;  // host copy of the last upload (launch descriptors, for merging plans)
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void ensure(size_t count) {
    if (count <= n && p) return;
    release();
    size_t bytes = sizeof(T) * (count ? count : 1);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      throw CudaError{e};
    }
    n = count;
  }
  void upload(const std::vector<T> &v) {
    h = v;
    ensure(v.size());
    if (!v.empty()) HODLR_CUDA_TRY(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  }
};

// Per-node factorization data kept for solves with the same factors.
struct NodeStore {
  DevBuf<double> S;      // form 0, per node: S = I - V1Tu1 V0Tu0 (r x r)
  DevBuf<double> F;      // per node: r x r FP64 work of the factor kernel
  DevBuf<double> ident;  // r x r identity (the I of S)
  DevBuf<double> M64;    // per node: (2r)^2 solve matrix, FP64 path
  DevBuf<float> M32;     // per node: (2r)^2 solve matrix, mixed path
  int rr = 0, mm = 0;
};

template <typename T, typename TE>
struct LevelPlan {
  DevBuf<GemmItem<T, T>> red_items;
  DevBuf<GemmSeg<T>> red_segs;
  int n_red = 0, red_max_m = 0, red_max_n = 0;
  int v_lo = 0, v_hi = 0;  // columns of V its reduce reads: [v_lo, v_hi)
  DevBuf<SumTask<T>> sums;          // partial slots -> one W per child
  int n_sums = 0;
  int sum_max_slots = 0;             // most partial slots of one of its tasks
  long long sum_max_len = 0;
  DevBuf<GemmItem<T, double>> gram_items;  // S = I - V1Tu1 V0Tu0, FP64 result
  DevBuf<GemmSeg<T>> gram_segs;
  int n_gram = 0, gram_max = 0;
  // node factorization tasks by form (0: r x r reduced system, 1: 2r x 2r
  // permuted Schur system of the nodes inside a Legion leaf)
  DevBuf<NodeTask<T, TE>> node_tasks[2];
  int n_nodes[2] = {0, 0}, max_s[2] = {0, 0}, max_r[2] = {0, 0};
  bool g_alias[2] = {false, false};  // node_g_alias of each form's tasks
  DevBuf<GemmItem<T, T>> ap_items;  // [eta0; eta1] = M [V0Td0; V1Td1] per node
  DevBuf<GemmSeg<T>> ap_segs;
  int n_ap = 0, ap_max_m = 0, ap_max_n = 0;
  DevBuf<GemmItem<T, T>> bc_items;
  DevBuf<GemmSeg<T>> bc_segs;
  int n_bc = 0, bc_max_m = 0, bc_max_n = 0;
};

// One batched GEMM launch: items + their segments.
template <typename TA, typename TC>
struct GemmLaunch {
  DevBuf<GemmItem<TA, TC>> items;
  DevBuf<GemmSeg<TA>> segs;
  int n = 0, max_m = 0, max_n = 0;
  void set(const std::vector<GemmItem<TA, TC>> &it, const std::vector<GemmSeg<TA>> &sg) {
    items.upload(it);
    segs.upload(sg);
    n = (int)it.size();
    max_m = max_n = 0;
    for (const auto &x : it) {
      max_m = max_m > x.M ? max_m : x.M;
      max_n = max_n > x.N ? max_n : x.N;
    }
  }
};

// Blocked factorization of every leaf on [D | X] (leaf_blocked.cu), two
// levels: outer blocks of `ob` columns, each factored as ob / nb register
// panels whose row interchanges and updates stay inside the block's columns;
// then the block's interchanges on the other columns, the block-row solve
// and one trailing update of depth ob.  The backward solve on X runs by the
// same blocks.  With ob <= 128 the block-row solves (forward on the rows of
// the block, backward on X) are single products with the inverses of the
// block's triangles, built from the panels' inverses; larger blocks solve
// panel by panel.  ob == nb is the one-level right-looking factorization.
template <typename T>
struct LeafPlan {
  DevBuf<LeafFactorTask<T>> tasks;
  DevBuf<T> Linv, Uinv;
  DevBuf<T> LinvB, UinvB;  // outer-block inverses (two-level plans with ob <= 128)
  DevBuf<int> swapflag;
  std::vector<LeafFactorTask<T>> host_tasks;  // for apply plans with these factors
  int nleaf = 0, max_n = 0, laswp_cols = 0, nb = 0, ob = 0;
  enum Kind { kPanel, kLaswp, kTrsm, kUpdate, kBlockInv };
  struct Step {
    Kind kind = kPanel;
    int k0 = 0, panel = 0;          // kPanel: the panel; kLaswp: first panel
    int block = 0;                  // kBlockInv: the outer block
    int np = 0;                     // kLaswp: panels applied
    int a0 = 0, a1 = 0, b0 = 0, b1 = 0;  // kLaswp: D column ranges (clamped per leaf)
    bool with_x = false;            // kLaswp: X columns too
    GemmLaunch<T, T> g;             // kTrsm (C = A B) / kUpdate (C -= A B)
  };
  // fwd: the steps of block 0, then block 1, ... (fwd_per_block each);
  // bwd: the steps of the last block first (bwd_per_block each)
  std::vector<std::unique_ptr<Step>> fwd, bwd;
  int nblocks = 0, fwd_per_block = 0, bwd_per_block = 0;
  bool binv = false;  // block rows solved with the outer blocks' inverses
};

template <typename T, typename TE>
struct PathPlan {
  bool built = false;
  bool factor = false;  // getrf + node factor (fused) vs getrs + node apply only
  DevBuf<LeafTask<T>> leaf_tasks;
  int nleaf = 0, max_n = 0, max_nrhs = 0;
  LeafPlan<T> leaf;     // factor paths: the blocked leaf factorization
  DevBuf<LeafFactorTask<T>> apply_tasks;  // apply paths: the factors' tasks on X
  int apply_nb = 0, apply_max_n = 0, apply_max_cols = 0;
  std::vector<std::unique_ptr<LevelPlan<T, TE>>> levels;  // deepest first
  // FP32 apply paths: the levels as one persistent launch (sweep.cu)
  DevBuf<SweepLevel> sweep;
  DevBuf<unsigned> sweep_bar;
  int sweep_max_n = 0;
  bool sweep_ok = false;
};

// Matvec plan: y = beta b + alpha (D x + sum_c U_c V_sib^T x_sib).
struct MatvecPlan {
  bool built = false;
  DevBuf<GemmItem<double, double>> red_items;
  DevBuf<GemmSeg<double>> red_segs;
  int n_red = 0, red_max_m = 0, red_max_n = 0;
  DevBuf<SumTask<double>> sums;
  int n_sums = 0;
  long long sum_max_len = 0;
  DevBuf<GemmItem<double, double>> ap_items;
  DevBuf<GemmSeg<double>> ap_segs;
  int n_ap = 0, ap_max_m = 0, ap_max_n = 0;
};

// Optional per-phase timing (CUDA events around each launch group).
enum Phase {
  PH_GETRF = 0, PH_GETRS, PH_REDUCE, PH_NODE_FACTOR, PH_NODE_APPLY, PH_BCAST, PH_MATVEC,
  PH_CONVERT, PH_LEAF_PANEL, PH_LEAF_UPDATE, PH_LEAF_TRSM, PH_SWEEP_LEVELS, PH_COUNT
};
struct Profiler {
  bool on = false;
  struct Rec { int phase; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  double ms[PH_COUNT] = {0};
  long long launches[PH_COUNT] = {0};
  void begin(int ph, cudaStream_t s, cudaEvent_t &a);
  void end(int ph, cudaStream_t s, cudaEvent_t a);
  void collect();  // sync + accumulate + free events
  void reset();
};

// A replayable segment of the solve captured once as a CUDA graph.  The
// segment only depends on the system's buffers (fixed after the first solve),
// so the captured graph stays valid for every later right-hand side or
// matrix loaded into the same buffers.
struct GraphSeg {
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;  // kernel launches recorded in the graph
  GraphSeg() = default;
  GraphSeg(const GraphSeg &) = delete;
  GraphSeg &operator=(const GraphSeg &) = delete;
  ~GraphSeg() { reset(); }
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    kernels = 0;
  }
};

// Runs `fn` (stream work on s) through the graph cache `g`: captured on the
// first call, replayed afterwards; eager when `eager` is set or on the legacy
// default stream (which cannot be captured).
template <typename F>
void run_graph(GraphSeg &g, bool eager, cudaStream_t s, F &&fn) {
  if (eager || s == nullptr) {
    fn();
    return;
  }
  if (!g.exec) {
    const long long before = launch_total();
    cudaGraph_t graph = nullptr;
    HODLR_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      fn();
    } catch (...) {
      cudaStreamEndCapture(s, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    HODLR_CUDA_TRY(cudaStreamEndCapture(s, &graph));
    cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      g.exec = nullptr;
      throw CudaError{e};
    }
    g.kernels = launch_total() - before;
    add_launches(-g.kernels);  // counted when replayed
  }
  HODLR_CUDA_TRY(cudaGraphLaunch(g.exec, s));
  add_launches(g.kernels);
}

// part masks of a path: the leaf solves / factorization and the tree levels
constexpr int kPathLeaves = 1, kPathLevels = 2;
// called before each level of a path, in order: (level index, the columns of
// V its reduce reads [v_lo, v_hi))
using LevelHook = std::function<void(int, int, int)>;

// A stream for copies of host input and two events on it, created on first
// use (hodlr_solve_refined_host)
struct CopyLane {
  cudaStream_t stream = nullptr;
  cudaEvent_t inputs = nullptr;  // D, B and U copied (recorded on the solve stream)
  cudaEvent_t v = nullptr;       // V copied (recorded on the copy stream)
  std::vector<cudaEvent_t> level_v;  // V's columns of level l copied
  CopyLane() = default;
  CopyLane(const CopyLane &) = delete;
  CopyLane &operator=(const CopyLane &) = delete;
  ~CopyLane() {
    for (cudaEvent_t e : level_v) cudaEventDestroy(e);
    if (inputs) cudaEventDestroy(inputs);
    if (v) cudaEventDestroy(v);
    if (stream) cudaStreamDestroy(stream);
  }
  void ensure() {
    if (!stream) HODLR_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    if (!inputs) HODLR_CUDA_TRY(cudaEventCreateWithFlags(&inputs, cudaEventDisableTiming));
    if (!v) HODLR_CUDA_TRY(cudaEventCreateWithFlags(&v, cudaEventDisableTiming));
  }
  void ensure_levels(size_t n) {
    while (level_v.size() < n) {
      cudaEvent_t e = nullptr;
      HODLR_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      level_v.push_back(e);
    }
  }
};

struct System {
  Tree tree;
  int N = 0, m = 0, r = 0, C = 0, vc = 0, nmax = 0;
  // originals (FP64)
  DevBuf<double> D, U, V, B, Xsol;
  // FP64 path
  DevBuf<double> X64, DLU64, Y64;
  DevBuf<int> ipiv64, perm64;
  // mixed path
  DevBuf<float> X32, D32, V32, Y32;
  DevBuf<int> ipiv32, perm32;
  DevBuf<double> R64, MVx, relres_dev, ratio_part;
  // workspaces
  DevBuf<double> part64, wfin64, eta64, tbuf, mvpart;
  DevBuf<float> part32, wfin32, eta32;
  DevBuf<int> info;
  NodeStore ns64, ns32;
  PathPlan<double, double> fused64[2];  // [form]
  PathPlan<double, double> apply64[2];
  PathPlan<float, float> fused32, apply32;
  MatvecPlan mv_sol, mv_usr;
  int factored = -1;  // HODLR_PREC_* of the current factorization, -1 none
  int factored_form = 0;
  int red_chunk = 512;
  int nb32 = 0;  // forced FP32 leaf panel width (0: by the largest leaf)
  int ob32 = 128, ob64 = 0;  // leaf outer block width per path (0: one level)
  int bc_chunk = 512;
  int n_info = 0;
  // granularity of the reference's tasks (HodlrMatrix leafSize): the FP64
  // fused path solves the nodes inside a Legion leaf with the 2r x 2r form
  int leaf_size = 1;
  Profiler prof;
  bool use_graphs = true;  // replay captured segments (off while profiling)
  GraphSeg g_factor32, g_sweep32, g_factor64, g_fused64[2], g_sweep64;
  GraphSeg g_factor32_leaves;  // the leaf part of run_factor32 (hodlr_solve_refined_host)
  CopyLane lane;  // copies of host input (hodlr_solve_refined_host)

  int init(int N_, int nrhs, int rank, int threshold);
  void ensure_fp64();
  void ensure_mixed();

  void run_fused64(int form, cudaStream_t s);     // X64 = [B|U], DLU64 = D, walk
  void run_apply64(cudaStream_t s);               // Y64 <- A^{-1} Y64 with fused64 factors
  void run_factor32(cudaStream_t s);              // X32 = f32([B|U]), D32 = f32(D), walk
  // one part of run_factor32 (kPathLeaves: conversion of D, [B|U] and the
  // leaf factorization; kPathLevels: conversion of V and the tree levels)
  void run_factor32_part(int parts, cudaStream_t s);
  // the levels part with `hook` before each level, V converted level by level
  // inside the hook's caller (run_factor32_levels_hooked)
  void run_factor32_levels_hooked(const LevelHook &hook, cudaStream_t s);
  void convert32(int parts, cudaStream_t s);      // the FP64 -> FP32 copies of those parts
  void convert_v32(int lo, int hi, cudaStream_t s);  // V32 = f32(V) for columns [lo, hi)
  void run_apply32(cudaStream_t s);               // Y32 <- A^{-1} Y32
  void run_matvec(const MatvecPlan &p, double alpha, double beta, cudaStream_t s);
  int check_info(cudaStream_t s);                 // sync + first nonzero INFO
  double relres(cudaStream_t s);                  // of Xsol against B (sync)
  void relres_enqueue(cudaStream_t s);            // matvec + column ratios into relres_dev
  double relres_read(cudaStream_t s);             // sync + max of relres_dev
  template <typename F>
  void run_graph(GraphSeg &g, cudaStream_t s, F &&fn) {
    ::hodlr::run_graph(g, !use_graphs || prof.on, s, fn);
  }
  void reset_graphs() {
    g_factor32.reset(); g_sweep32.reset(); g_factor64.reset(); g_sweep64.reset();
    g_factor32_leaves.reset();
    g_fused64[0].reset(); g_fused64[1].reset();
  }
};

// Many independent systems of uneven size, rank and right-hand-side count
// solved together: their level schedules are merged step by step (every
// leaf panel of every system in one launch, then each system's deepest
// remaining level in one launch per phase, ...), so the batch costs one
// launch per tree level and phase rather than one per system.  Mixed
// precision with FP64 refinement; every system keeps its own buffers and
// factors, and the merged plans only hold launch descriptors that point into
// them.  The systems must outlive the batch and keep their sizes.
struct Batch {
  std::vector<System *> sys;
  // Systems whose merged walk shares kernels: same FP32 leaf panel width and
  // the same right-hand-side class (<= 16 or more columns: the skinny
  // kernels' column tile).  Groups run back to back.
  struct Group {
    int nb = 0, ob = 0;
    bool wide = false;
    std::vector<int> members;
    PathPlan<float, float> fused32, apply32;
  };
  std::vector<std::unique_ptr<Group>> groups;
  MatvecPlan mv;
  DevBuf<Ew2DTask<double, float>> cv_in, cv_res;  // D, B, U, V -> FP32; R64 -> Y32
  DevBuf<Ew2DTask<float, double>> cv_x0, add_y;   // X32 -> Xsol; Xsol += Y32
  long long t_in = 0, t_res = 0, t_x0 = 0;        // total tiles of each pass
  DevBuf<RatioTask> ratios;
  int max_m = 0;
  DevBuf<double> rr;            // column residual ratios, system k at rr_off[k]
  std::vector<int> rr_off;
  DevBuf<int> info;             // all systems' INFO slots, system k at info_off[k]
  std::vector<int> info_off;
  int n_info = 0;
  bool use_graphs = true;
  GraphSeg g_factor, g_sweep;
  Profiler prof;
  void build(const std::vector<System *> &systems);
  void run_factor(cudaStream_t s);   // conversions, merged walk, x0, residuals
  void run_sweep(cudaStream_t s);    // one refinement sweep of every system, residuals
  void residuals(cudaStream_t s);    // merged matvec R = B - A Xsol + column ratios
  // sync; the first nonzero INFO (leaf code, or 100000 + node code) and its system
  int check_info(cudaStream_t s, int *failed);
  // sync; the largest ratio, and each system's largest in per_system
  double relres_read(cudaStream_t s, std::vector<double> *per_system);
  template <typename F>
  void run_graph(GraphSeg &g, cudaStream_t s, F &&fn) {
    ::hodlr::run_graph(g, !use_graphs || prof.on, s, fn);
  }
};

}  // namespace hodlr

// The C ABI's opaque handles (include/hodlr_gpu.h).
struct hodlr_system_s {
  hodlr::System sys;
};
struct hodlr_batch_s {
  hodlr::Batch b;
};
