// capi.cu -- the extern "C" entry points declared in include/hodlr_gpu.h.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "gemm_simt.cuh"
#include "leaf.cuh"
#include "node.cuh"
#include "solver.h"
#include "tc_gemm.cuh"
#include "util.cuh"

namespace hodlr {

namespace {
thread_local long long g_launches = 0;
}

void count_launch() { ++g_launches; }
void add_launches(long long n) { g_launches += n; }
long long launch_total() { return g_launches; }

void raise_smem_limit(const void *func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> set;  // (function, device) -> limit
  int dev = 0;
  HODLR_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  size_t &cur = set[std::make_pair(func, dev)];
  if (bytes <= cur) return;
  HODLR_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bytes));
  cur = bytes;
}

}  // namespace hodlr

using namespace hodlr;


namespace {

// Runs `f` and maps library exceptions to status codes.
template <typename F>
int guarded(F &&f) {
  try {
    return f();
  } catch (const CudaError &e) {
    return e.err == cudaErrorMemoryAllocation ? HODLR_ERR_NOMEM : HODLR_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    return HODLR_ERR_NOMEM;
  }
}

int device_ok() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return HODLR_ERR_CUDA;
  }
  return 0;
}

// Small stream-ordered device scratch for single-call task bodies.
struct StreamScratch {
  void *p = nullptr;
  cudaStream_t s;
  explicit StreamScratch(size_t bytes, cudaStream_t st) : s(st) {
    HODLR_CUDA_TRY(cudaMallocAsync(&p, bytes, s));
  }
  ~StreamScratch() {
    if (p) cudaFreeAsync(p, s);
  }
};

// HODLR_ERR_TIMEOUT if a tensor-core kernel's bounded wait gave up since the
// flag was last read (the flag is sticky per device until read), else 0.
// Call after the work has been synchronized.
int tc_status() {
  const bool tc = tc_error_flag(true) > 0;
  const bool sw = sweep_error_flag(true) > 0;
  return (tc || sw) ? HODLR_ERR_TIMEOUT : 0;
}

int finish_info(int *info_user, int *info_dev, cudaStream_t s) {
  if (info_user) return 0;
  int h = 0;
  HODLR_CUDA_TRY(cudaMemcpyAsync(&h, info_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
  HODLR_CUDA_TRY(cudaStreamSynchronize(s));
  return h;
}

}  // namespace

extern "C" {

long long hodlr_launch_count(void) { return g_launches; }
void hodlr_reset_launch_count(void) { g_launches = 0; }

const char *hodlr_status_string(int status) {
  switch (status) {
    case HODLR_OK: return "ok";
    case HODLR_ERR_CUDA: return "CUDA runtime error or no CUDA device";
    case HODLR_ERR_NOMEM: return "device allocation failed";
    case HODLR_ERR_STATE: return "call out of order";
    case HODLR_ERR_NOCONV: return "refinement did not reach the tolerance";
    case HODLR_ERR_TIMEOUT: return "bounded device wait gave up";
    case HODLR_ERR_UNSUPPORTED: return "unsupported size or option";
    case HODLR_ERR_IO: return "file could not be opened, read or written";
    default: break;
  }
  if (status > 0) return "zero pivot (LAPACK-style INFO)";
  return "invalid argument";
}

// ---------------------------------------------------------------------------
// task bodies
// ---------------------------------------------------------------------------

int hodlr_leaf_solve(int n, int nrhs, double *D, int ldd, double *X, int ldx, int *ipiv,
                     int *info, hodlr_stream_t stream) {
  if (n < 0) return -1;
  if (nrhs < 0) return -2;
  if (!D && n > 0) return -3;
  if (ldd < (n > 1 ? n : 1)) return -4;
  if (!X && n > 0 && nrhs > 0) return -5;
  if (ldx < (n > 1 ? n : 1)) return -6;
  if (!ipiv && n > 0) return -7;
  if (n > 1024) return HODLR_ERR_UNSUPPORTED;
  if (int e = device_ok()) return e;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    if (n == 0) return 0;
    StreamScratch scr(sizeof(int), s);
    int *info_dev = info ? info : static_cast<int *>(scr.p);
    LeafTask<double> tk{};
    tk.D = D; tk.ldd = ldd; tk.X = X; tk.ldx = ldx; tk.ipiv = ipiv; tk.perm = nullptr;
    tk.n = n; tk.nrhs = nrhs; tk.info_slot = 0;
    launch_getrf<double>(nullptr, tk, 1, n, info_dev, s);
    if (nrhs > 0) launch_getrs<double>(nullptr, tk, 1, n, nrhs, s);
    return finish_info(info, info_dev, s);
  });
}

int hodlr_leaf_solve_batched(int count, const hodlr_leaf_desc *descs, int max_n, int max_nrhs,
                             int *info, hodlr_stream_t stream) {
  if (count < 0) return -1;
  if (!descs && count > 0) return -2;
  if (max_n < 0 || max_n > 1024) return max_n < 0 ? -3 : HODLR_ERR_UNSUPPORTED;
  if (max_nrhs < 0) return -4;
  if (!info && count > 0) return -5;
  if (int e = device_ok()) return e;
  static_assert(sizeof(hodlr_leaf_desc) == sizeof(LeafTask<double>) - 2 * sizeof(int),
                "descriptor layout");
  return guarded([&]() -> int {
    if (count == 0) return 0;
    cudaStream_t s = as_stream(stream);
    // hodlr_leaf_desc has no info_slot: expand into LeafTask on the device
    std::vector<hodlr_leaf_desc> h(count);
    HODLR_CUDA_TRY(cudaMemcpyAsync(h.data(), descs, sizeof(hodlr_leaf_desc) * count,
                                   cudaMemcpyDeviceToHost, s));
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<LeafTask<double>> t(count);
    for (int i = 0; i < count; ++i) {
      t[i].D = h[i].D; t[i].X = h[i].X; t[i].ipiv = h[i].ipiv; t[i].perm = h[i].perm;
      t[i].ldd = h[i].ldd; t[i].ldx = h[i].ldx; t[i].n = h[i].n; t[i].nrhs = h[i].nrhs;
      t[i].info_slot = i;
      if (h[i].n > max_n || h[i].nrhs > max_nrhs || h[i].ldd < h[i].n || h[i].ldx < h[i].n)
        return -2;
    }
    StreamScratch scr(sizeof(LeafTask<double>) * count, s);
    HODLR_CUDA_TRY(cudaMemcpyAsync(scr.p, t.data(), sizeof(LeafTask<double>) * count,
                                   cudaMemcpyHostToDevice, s));
    LeafTask<double> none{};
    auto *tp = static_cast<LeafTask<double> *>(scr.p);
    launch_getrf<double>(tp, none, count, max_n, info, s);
    launch_getrs<double>(tp, none, count, max_n, max_nrhs, s);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  });
}

int hodlr_gemm_reduce(double alpha, int k, int r, int ncol, const double *V, int ldv,
                      const double *U, int ldu, int col_beg, double *W, int ldw,
                      hodlr_stream_t stream) {
  if (k < 0) return -2;
  if (r < 0) return -3;
  if (ncol < 0) return -4;
  if (!V && k > 0 && r > 0) return -5;
  if (ldv < (k > 1 ? k : 1)) return -6;
  if (!U && k > 0 && ncol > 0) return -7;
  if (ldu < (k > 1 ? k : 1)) return -8;
  if (col_beg < 0) return -9;
  if (!W && r > 0 && ncol > 0) return -10;
  if (ldw < (r > 1 ? r : 1)) return -11;
  if (int e = device_ok()) return e;
  return guarded([&]() -> int {
    if (r == 0 || ncol == 0) return 0;
    cudaStream_t s = as_stream(stream);
    // split K into row chunks: partials in scratch, then W += sum (fixed order)
    const int chunk = 4096;
    const int nsl = k > 0 ? cdiv(k, chunk) : 0;
    if (nsl == 0) return 0;
    std::vector<GemmItem<double, double>> it(nsl);
    std::vector<GemmSeg<double>> sg(nsl);
    const size_t slot = (size_t)r * ncol;
    StreamScratch part(sizeof(double) * slot * nsl, s);
    double *pp = static_cast<double *>(part.p);
    for (int q = 0; q < nsl; ++q) {
      const int rb = q * chunk, rows = std::min(chunk, k - rb);
      sg[q] = GemmSeg<double>{V + rb, U + rb + (long long)col_beg * ldu, ldv, ldu, rows, 0};
      it[q] = GemmItem<double, double>{pp + q * slot, nullptr, r, 0, r, ncol, q, 1};
    }
    StreamScratch desc(sizeof(GemmItem<double, double>) * nsl + sizeof(GemmSeg<double>) * nsl +
                           2 * sizeof(GemmItem<double, double>) + sizeof(SumTask<double>) + 256,
                       s);
    auto *di = static_cast<GemmItem<double, double> *>(desc.p);
    auto *ds = reinterpret_cast<GemmSeg<double> *>(di + nsl);
    HODLR_CUDA_TRY(cudaMemcpyAsync(di, it.data(), sizeof(it[0]) * nsl, cudaMemcpyHostToDevice, s));
    HODLR_CUDA_TRY(cudaMemcpyAsync(ds, sg.data(), sizeof(sg[0]) * nsl, cudaMemcpyHostToDevice, s));
    launch_gemm_items<double, double, double>(di, ds, nsl, r, ncol, true, alpha, 0.0, s);
    // W += fixed-order sum of the partials
    SumTask<double> st{};
    StreamScratch tmp(sizeof(double) * slot, s);
    st.dst = static_cast<double *>(tmp.p);
    st.src = pp;
    st.len = (long long)slot;
    st.stride = (long long)slot;
    st.nslots = nsl;
    auto *dst = reinterpret_cast<SumTask<double> *>(ds + nsl);
    HODLR_CUDA_TRY(cudaMemcpyAsync(dst, &st, sizeof(st), cudaMemcpyHostToDevice, s));
    launch_sum_slots<double>(dst, 1, st.len, s);
    launch_add2d<double>(W, ldw, static_cast<double *>(tmp.p), r, r, ncol, s);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  });
}

int hodlr_gemm_f32(int transa, int m, int n, int k, float alpha, const float *A, int lda,
                   const float *B, int ldb, float beta, float *C, int ldc, int engine,
                   hodlr_stream_t stream) {
  if (transa != 0 && transa != 1) return -1;
  if (m < 0) return -2;
  if (n < 0) return -3;
  if (k < 0) return -4;
  if (!A && m > 0 && k > 0) return -6;
  if (lda < std::max(1, transa ? k : m)) return -7;
  if (!B && k > 0 && n > 0) return -8;
  if (ldb < std::max(1, k)) return -9;
  if (!C && m > 0 && n > 0) return -11;
  if (ldc < std::max(1, m)) return -12;
  if (engine != 0 && engine != 1) return -13;
  if (int e = device_ok()) return e;
  return guarded([&]() -> int {
    if (m == 0 || n == 0) return 0;
    cudaStream_t s = as_stream(stream);
    GemmSeg<float> sg{A, B, lda, ldb, k, 0};
    GemmItem<float, float> it{C, C, ldc, ldc, m, n, 0, 1};
    StreamScratch scr(sizeof(sg) + sizeof(it) + 64, s);
    auto *di = static_cast<GemmItem<float, float> *>(scr.p);
    auto *ds = reinterpret_cast<GemmSeg<float> *>(di + 1);
    HODLR_CUDA_TRY(cudaMemcpyAsync(di, &it, sizeof(it), cudaMemcpyHostToDevice, s));
    HODLR_CUDA_TRY(cudaMemcpyAsync(ds, &sg, sizeof(sg), cudaMemcpyHostToDevice, s));
    if (engine == 1)
      launch_tc_gemm<float>(di, ds, 1, m, n, transa != 0, alpha, beta, s);
    else
      launch_gemm_items<float, float, float>(di, ds, 1, m, n, transa != 0, alpha, beta, s, false);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return tc_status();
  });
}

int hodlr_debug_sweep_barrier_hook(long long polls, int skip_one_arrival) {
  if (int e = device_ok()) return e;
  return guarded([&]() -> int {
    HODLR_CUDA_TRY(cudaDeviceSynchronize());
    sweep_set_wait_hook(polls, skip_one_arrival);
    return 0;
  });
}

int hodlr_debug_tc_wait_hook(long long polls, int skip_one_commit) {
  if (int e = device_ok()) return e;
  return guarded([&]() -> int {
    HODLR_CUDA_TRY(cudaDeviceSynchronize());
    tc_set_wait_hook(polls, skip_one_commit);
    return 0;
  });
}

static int node_solve_common(int form, int r0, int r1, int c, const double *V0Tu0, int ld00,
                             const double *V1Tu1, int ld11, double *V0Td0, int ld0d,
                             double *V1Td1, int ld1d, int *info, hodlr_stream_t stream) {
  if (r0 <= 0) return -1;
  if (r1 <= 0) return -2;
  if (c < 0) return -3;
  if (!V0Tu0) return -4;
  if (ld00 < r1) return -5;
  if (!V1Tu1) return -6;
  if (ld11 < r0) return -7;
  if (!V0Td0 && c > 0) return -8;
  if (ld0d < r1) return -9;
  if (!V1Td1 && c > 0) return -10;
  if (ld1d < r0) return -11;
  const int s_ = form == 0 ? r0 : r0 + r1;
  if (form == 1 && r0 != r1) return HODLR_ERR_UNSUPPORTED;
  if (s_ > kMaxNodeS) return HODLR_ERR_UNSUPPORTED;
  if (int e = device_ok()) return e;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    // scratch: task | S (r0 x r0) | F (r1 x r0) | I (r0 x r0) | M (s2 x s2) | eta (s2 x c)
    //          | info | gram item + segment | apply item + 2 segments
    const int s2 = r0 + r1;
    const size_t nR = (size_t)r0 * r0, nF = (size_t)r1 * r0, nM = (size_t)s2 * s2;
    const size_t nE = (size_t)s2 * (c > 0 ? c : 1);
    const size_t need = 256 + sizeof(double) * (2 * nR + nF + nM + nE) + 8 * sizeof(int) + 1024;
    StreamScratch scr(need, s);
    char *base = static_cast<char *>(scr.p);
    auto *task = reinterpret_cast<NodeTask<double, double> *>(base);
    double *S = reinterpret_cast<double *>(base + 256);
    double *F = S + nR;
    double *ident = F + nF;
    double *M = ident + nR;
    double *eta = M + nM;
    int *info_dev = reinterpret_cast<int *>(eta + nE);
    auto *gitem = reinterpret_cast<GemmItem<double, double> *>(
        (reinterpret_cast<uintptr_t>(info_dev + 8) + 15) & ~uintptr_t(15));
    auto *gseg = reinterpret_cast<GemmSeg<double> *>(gitem + 1);
    auto *aitem = reinterpret_cast<GemmItem<double, double> *>(gseg + 1);
    auto *aseg = reinterpret_cast<GemmSeg<double> *>(aitem + 1);
    NodeTask<double, double> k{};
    k.W0u = V0Tu0; k.W1u = V1Tu1; k.ldw0u = ld00; k.ldw1u = ld11;
    k.S = S; k.F = F; k.M = M;
    k.r0 = r0; k.r1 = r1; k.info_slot = 0;
    HODLR_CUDA_TRY(cudaMemcpyAsync(task, &k, sizeof(k), cudaMemcpyHostToDevice, s));
    std::vector<double> I(nR, 0.0);
    for (int i = 0; i < r0; ++i) I[(size_t)i * r0 + i] = 1.0;
    GemmSeg<double> g{V1Tu1, V0Tu0, ld11, ld00, r1, 0};
    GemmItem<double, double> git{S, ident, r0, r0, r0, r0, 0, 1};
    GemmSeg<double> a2[2] = {{M, V0Td0, s2, ld0d, r1, 0},
                             {M + (size_t)r1 * s2, V1Td1, s2, ld1d, r0, 0}};
    GemmItem<double, double> ait{eta, nullptr, s2, 0, s2, c, 0, 2};
    if (form == 0) {
      // S = I - V1Tu1 V0Tu0 (the dgemm at solver_tasks.cc:261)
      HODLR_CUDA_TRY(cudaMemcpyAsync(ident, I.data(), sizeof(double) * nR, cudaMemcpyHostToDevice, s));
      HODLR_CUDA_TRY(cudaMemcpyAsync(gitem, &git, sizeof(git), cudaMemcpyHostToDevice, s));
      HODLR_CUDA_TRY(cudaMemcpyAsync(gseg, &g, sizeof(g), cudaMemcpyHostToDevice, s));
      launch_gemm_items<double, double, double>(gitem, gseg, 1, r0, r0, false, -1.0, 1.0, s);
    }
    HODLR_CUDA_TRY(cudaMemcpyAsync(aitem, &ait, sizeof(ait), cudaMemcpyHostToDevice, s));
    HODLR_CUDA_TRY(cudaMemcpyAsync(aseg, a2, sizeof(a2), cudaMemcpyHostToDevice, s));
    launch_node_factor<double, double>(task, 1, form == 0 ? r0 : s2, r0 > r1 ? r0 : r1, form,
                                       info_dev, s);
    int hinfo = 0;
    HODLR_CUDA_TRY(cudaMemcpyAsync(&hinfo, info_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));  // also ends the host staging buffers' use
    if (info) HODLR_CUDA_TRY(cudaMemcpyAsync(info, info_dev, sizeof(int), cudaMemcpyDeviceToDevice, s));
    if (hinfo == 0 && c > 0) {
      launch_gemm_items<double, double, double>(aitem, aseg, 1, s2, c, false, 1.0, 0.0, s);
      // outputs in place: form 0 writes eta0 over V1Td1, eta1 over V0Td0
      // (fast_solver.cc:238-240); form 1 eta0 over V0Td0, eta1 over V1Td1.
      double *o0 = form == 0 ? V1Td1 : V0Td0;
      double *o1 = form == 0 ? V0Td0 : V1Td1;
      const int l0 = form == 0 ? ld1d : ld0d, l1 = form == 0 ? ld0d : ld1d;
      HODLR_CUDA_TRY(cudaMemcpy2DAsync(o0, sizeof(double) * l0, eta, sizeof(double) * s2,
                                       sizeof(double) * r0, c, cudaMemcpyDeviceToDevice, s));
      HODLR_CUDA_TRY(cudaMemcpy2DAsync(o1, sizeof(double) * l1, eta + r0, sizeof(double) * s2,
                                       sizeof(double) * r1, c, cudaMemcpyDeviceToDevice, s));
    }
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));  // scratch lifetime
    return info ? 0 : hinfo;  // with a device INFO pointer the value goes there
  });
}

int hodlr_node_lu_solve(int r0, int r1, int c, const double *V0Tu0, int ld00,
                        const double *V1Tu1, int ld11, double *V0Td0, int ld0d, double *V1Td1,
                        int ld1d, int *info, hodlr_stream_t stream) {
  return node_solve_common(0, r0, r1, c, V0Tu0, ld00, V1Tu1, ld11, V0Td0, ld0d, V1Td1, ld1d,
                           info, stream);
}

int hodlr_node_schur2_solve(int r0, int r1, int c, const double *V0Tu0, int ld00,
                            const double *V1Tu1, int ld11, double *V0Td0, int ld0d,
                            double *V1Td1, int ld1d, int *info, hodlr_stream_t stream) {
  return node_solve_common(1, r0, r1, c, V0Tu0, ld00, V1Tu1, ld11, V0Td0, ld0d, V1Td1, ld1d,
                           info, stream);
}

int hodlr_gemm_broadcast(double alpha, double beta, int k, int r, int c, double *X, int ldx,
                         int u_col_beg, const double *eta, int lde, int d_col_beg,
                         hodlr_stream_t stream) {
  if (k < 0) return -3;
  if (r < 0) return -4;
  if (c < 0) return -5;
  if (!X && k > 0) return -6;
  if (ldx < (k > 1 ? k : 1)) return -7;
  if (u_col_beg < 0) return -8;
  if (!eta && r > 0 && c > 0) return -9;
  if (lde < (r > 1 ? r : 1)) return -10;
  if (d_col_beg < 0) return -11;
  if (!(u_col_beg + r <= d_col_beg || d_col_beg + c <= u_col_beg)) return -11;
  if (int e = device_ok()) return e;
  return guarded([&]() -> int {
    if (k == 0 || c == 0) return 0;
    cudaStream_t s = as_stream(stream);
    GemmSeg<double> sg{X + (long long)u_col_beg * ldx, eta, ldx, lde, r, 0};
    double *Cp = X + (long long)d_col_beg * ldx;
    GemmItem<double, double> it{Cp, Cp, ldx, ldx, k, c, 0, 1};
    StreamScratch scr(sizeof(sg) + sizeof(it) + 64, s);
    auto *di = static_cast<GemmItem<double, double> *>(scr.p);
    auto *ds = reinterpret_cast<GemmSeg<double> *>(di + 1);
    HODLR_CUDA_TRY(cudaMemcpyAsync(di, &it, sizeof(it), cudaMemcpyHostToDevice, s));
    HODLR_CUDA_TRY(cudaMemcpyAsync(ds, &sg, sizeof(sg), cudaMemcpyHostToDevice, s));
    launch_gemm_items<double, double, double>(di, ds, 1, k, c, false, alpha, beta, s);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  });
}

// ---------------------------------------------------------------------------
// handle API
// ---------------------------------------------------------------------------

int hodlr_build_tree(int N, int nrhs, int rank, int threshold, int *out, int cap) {
  Tree t;
  const int rc = build_tree(N, nrhs, rank, threshold, t);
  if (rc < 0) return rc;
  if (!out || cap < (int)t.nodes.size()) return -6;
  std::memcpy(out, t.nodes.data(), sizeof(Node) * t.nodes.size());
  return (int)t.nodes.size();
}

int hodlr_create(hodlr_system *out, int N, int nrhs, int rank, int threshold) {
  if (!out) return -1;
  *out = nullptr;
  if (N <= 0) return -2;
  if (nrhs <= 0) return -3;
  if (rank <= 0) return -4;
  if (threshold <= 0) return -5;
  if (rank > kMaxNodeS) return HODLR_ERR_UNSUPPORTED;
  if (int e = device_ok()) return e;
  auto *h = new (std::nothrow) hodlr_system_s;
  if (!h) return HODLR_ERR_NOMEM;
  int rc = guarded([&]() -> int {
    int t = h->sys.init(N, nrhs, rank, threshold);
    if (t < 0) return t - 1;  // -1..-4 of build_tree -> argument positions 2..5
    if (h->sys.nmax > 1024) return HODLR_ERR_UNSUPPORTED;
    return 0;
  });
  if (rc != 0) {
    delete h;
    return rc;
  }
  *out = h;
  return 0;
}

int hodlr_destroy(hodlr_system sys) {
  if (!sys) return -1;
  delete sys;
  return 0;
}

int hodlr_tree_info(hodlr_system h, int *nnodes, int *max_depth, int *nleaves, int *ncols,
                    int *max_leaf) {
  if (!h) return -1;
  const Tree &t = h->sys.tree;
  if (nnodes) *nnodes = (int)t.nodes.size();
  if (max_depth) *max_depth = t.max_depth;
  if (nleaves) *nleaves = (int)t.leaves.size();
  if (ncols) *ncols = t.ncols;
  if (max_leaf) *max_leaf = t.max_leaf;
  return 0;
}

int hodlr_tree_nodes(hodlr_system h, int *out, int cap) {
  if (!h) return -1;
  const Tree &t = h->sys.tree;
  if (!out || cap < (int)t.nodes.size()) return -2;
  std::memcpy(out, t.nodes.data(), sizeof(Node) * t.nodes.size());
  return 0;
}

static int copy2d(double *dst, long long ldd, const double *src, long long lds, long long rows,
                  long long cols, int host, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return 0;
  HODLR_CUDA_TRY(cudaMemcpy2DAsync(dst, sizeof(double) * ldd, src, sizeof(double) * lds,
                                   sizeof(double) * rows, cols,
                                   host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  return 0;
}

int hodlr_set_matrix(hodlr_system h, const double *D, long long ldd, const double *U,
                     long long ldu, const double *V, long long ldv, int host,
                     hodlr_stream_t stream) {
  if (!h) return -1;
  System &S = h->sys;
  if (D && ldd < S.N) return -3;
  if (U && ldu < S.N) return -5;
  if (V && ldv < S.N) return -7;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    if (D) copy2d(S.D.p, S.N, D, ldd, S.N, S.nmax, host, s);
    if (U) copy2d(S.U.p, S.N, U, ldu, S.N, S.vc, host, s);
    if (V) copy2d(S.V.p, S.N, V, ldv, S.N, S.vc, host, s);
    if (host) HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    S.factored = -1;
    return 0;
  });
}

int hodlr_set_rhs(hodlr_system h, const double *B, long long ldb, int host,
                  hodlr_stream_t stream) {
  if (!h) return -1;
  System &S = h->sys;
  if (!B) return -2;
  if (ldb < S.N) return -3;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    copy2d(S.B.p, S.N, B, ldb, S.N, S.m, host, s);
    if (host) HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  });
}

int hodlr_get_matrix(hodlr_system h, double *D, long long ldd, double *U, long long ldu,
                     double *V, long long ldv, double *B, long long ldb, int host,
                     hodlr_stream_t stream) {
  if (!h) return -1;
  System &S = h->sys;
  if (D && ldd < S.N) return -3;
  if (U && ldu < S.N) return -5;
  if (V && ldv < S.N) return -7;
  if (B && ldb < S.N) return -9;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    const cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    auto out = [&](double *dst, long long ld, const double *src, long long cols) {
      if (!dst || cols <= 0) return;
      HODLR_CUDA_TRY(cudaMemcpy2DAsync(dst, sizeof(double) * ld, src, sizeof(double) * S.N,
                                       sizeof(double) * S.N, cols, k, s));
    };
    out(D, ldd, S.D.p, S.nmax);
    out(U, ldu, S.U.p, S.vc);
    out(V, ldv, S.V.p, S.vc);
    out(B, ldb, S.B.p, S.m);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  });
}

// (row_beg, rows) of every Legion leaf, left to right
static std::vector<int2> legion_leaf_ranges(const System &S) {
  std::vector<int2> v;
  for (int id : legion_leaves(S.tree, S.leaf_size))
    v.push_back(make_int2(S.tree.nodes[id].row_beg, S.tree.nodes[id].nrow));
  return v;
}

static std::vector<int2> leaf_ranges(const Tree &t) {
  std::vector<int2> v;
  for (int id : t.leaves) v.push_back(make_int2(t.nodes[id].row_beg, t.nodes[id].nrow));
  return v;
}

int hodlr_init_circulant(hodlr_system h, double diag, hodlr_stream_t stream) {
  if (!h) return -1;
  return guarded([&]() -> int {
    System &S = h->sys;
    cudaStream_t s = as_stream(stream);
    DevBuf<int2> lv;
    lv.upload(leaf_ranges(S.tree));
    HODLR_CUDA_TRY(cudaMemsetAsync(S.D.p, 0, sizeof(double) * (size_t)S.N * S.nmax, s));
    launch_circulant_k(lv.p, (int)S.tree.leaves.size(), S.nmax, S.D.p, S.N, S.r, diag, s);
    launch_circulant_uv(S.U.p, S.N, S.V.p, S.N, S.N, S.vc, S.r, s);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    S.factored = -1;
    return 0;
  });
}

int hodlr_init_rhs_drand48(hodlr_system h, long seed, hodlr_stream_t stream) {
  if (!h) return -1;
  return guarded([&]() -> int {
    System &S = h->sys;
    cudaStream_t s = as_stream(stream);
    DevBuf<int2> lv;
    const std::vector<int2> ranges = legion_leaf_ranges(S);
    lv.upload(ranges);
    launch_drand48(lv.p, (int)ranges.size(), S.B.p, S.N, S.m, seed, s);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  });
}

int hodlr_init_gaussian(hodlr_system h, unsigned long long seed, double offdiag_norm,
                        hodlr_stream_t stream) {
  if (!h) return -1;
  if (!(offdiag_norm > 0.0)) return -3;
  return guarded([&]() -> int {
    System &S = h->sys;
    const Tree &t = S.tree;
    cudaStream_t s = as_stream(stream);
    const long long N = S.N;
    const int m = S.m;
    HODLR_CUDA_TRY(cudaMemsetAsync(S.D.p, 0, sizeof(double) * (size_t)N * S.nmax, s));
    std::vector<FillTask> fills;
    long long fmax = 0;
    auto add_fill = [&](double *a, int rows, int cols, unsigned sid, double sc, double dg) {
      FillTask f{};
      f.a = a; f.lda = N; f.rows = rows; f.cols = cols; f.stream_id = sid;
      f.scale = sc; f.diag_add = dg;
      fills.push_back(f);
      fmax = std::max(fmax, (long long)rows * cols);
    };
    for (size_t q = 0; q < t.leaves.size(); ++q) {
      const Node &n = t.nodes[t.leaves[q]];
      add_fill(S.D.p + n.row_beg, n.nrow, n.nrow, (unsigned)(1 + q),
               1.0 / std::sqrt((double)n.nrow), 2.0);
    }
    const unsigned base = (unsigned)(1 + t.leaves.size());
    for (size_t i = 1; i < t.nodes.size(); ++i) {
      const Node &c = t.nodes[i];
      const double sc = 1.0 / std::sqrt((double)c.ncol * c.nrow);
      add_fill(S.U.p + c.row_beg + (long long)(c.col_beg - m) * N, c.nrow, c.ncol,
               base + 2 * (unsigned)i, sc, 0.0);
      add_fill(S.V.p + c.row_beg + (long long)(c.col_beg - m) * N, c.nrow, c.vncol,
               base + 2 * (unsigned)i + 1, sc, 0.0);
    }
    add_fill(S.B.p, (int)N, m, base + 2 * (unsigned)t.nodes.size() + 2, 1.0, 0.0);
    {
      DevBuf<FillTask> df;
      df.upload(fills);
      launch_gauss_fill_batched(df.p, (int)fills.size(), fmax, seed, s);
      HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    }
    // Rescale each off-diagonal block U_c V_s^T to spectral norm offdiag_norm:
    // ||U V^T||_2^2 = lambda_max((U^T U)(V^T V)); Grams via chunked reduces.
    std::vector<int> ids;
    for (size_t i = 1; i < t.nodes.size(); ++i) ids.push_back((int)i);
    const int r = S.r;
    const int chunk = 4096;
    std::vector<GemmItem<double, double>> it;
    std::vector<GemmSeg<double>> sg;
    std::vector<SumTask<double>> st;
    size_t nslot_total = 0;
    for (int i : ids) nslot_total += 2 * (size_t)cdiv(t.nodes[i].nrow, chunk);
    DevBuf<double> part, gram;
    part.ensure(nslot_total * r * r);
    gram.ensure(2 * ids.size() * (size_t)r * r);
    size_t slot = 0;
    for (size_t q = 0; q < ids.size(); ++q) {
      const Node &c = t.nodes[ids[q]];
      for (int which = 0; which < 2; ++which) {
        const double *A = (which == 0 ? S.U.p : S.V.p) + c.row_beg + (long long)(c.col_beg - m) * N;
        const int ns = cdiv(c.nrow, chunk);
        SumTask<double> sk{};
        sk.dst = gram.p + (2 * q + which) * (size_t)r * r;
        sk.src = part.p + slot * r * r;
        sk.len = (long long)r * r;
        sk.stride = (long long)r * r;
        sk.nslots = ns;
        st.push_back(sk);
        for (int z = 0; z < ns; ++z) {
          const int rb = z * chunk, rows = std::min(chunk, c.nrow - rb);
          sg.push_back(GemmSeg<double>{A + rb, A + rb, N, N, rows, 0});
          it.push_back(GemmItem<double, double>{part.p + (slot + z) * r * r, nullptr, r, 0, r, r,
                                                (int)sg.size() - 1, 1});
        }
        slot += ns;
      }
    }
    DevBuf<GemmItem<double, double>> dit;
    DevBuf<GemmSeg<double>> dsg;
    DevBuf<SumTask<double>> dst;
    dit.upload(it);
    dsg.upload(sg);
    dst.upload(st);
    launch_gemm_items<double, double, double>(dit.p, dsg.p, (int)it.size(), r, r, true, 1.0, 0.0,
                                              s);
    launch_sum_slots<double>(dst.p, (int)st.size(), (long long)r * r, s);
    std::vector<double> G(2 * ids.size() * (size_t)r * r);
    HODLR_CUDA_TRY(cudaMemcpyAsync(G.data(), gram.p, sizeof(double) * G.size(),
                                   cudaMemcpyDeviceToHost, s));
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    // index of node id in ids
    std::vector<int> pos(t.nodes.size(), -1);
    for (size_t q = 0; q < ids.size(); ++q) pos[ids[q]] = (int)q;
    std::vector<double> scale_u(t.nodes.size(), 1.0), scale_v(t.nodes.size(), 1.0);
    std::vector<double> v(r), w(r), z(r);
    for (size_t pi = 0; pi < t.nodes.size(); ++pi) {
      const Node &P = t.nodes[pi];
      if (P.is_leaf) continue;
      const int kids[2] = {P.lchild, P.rchild};
      for (int side = 0; side < 2; ++side) {
        const int c = kids[side], sb = kids[1 - side];
        const double *Gu = G.data() + (2 * (size_t)pos[c] + 0) * r * r;
        const double *Gv = G.data() + (2 * (size_t)pos[sb] + 1) * r * r;
        // power iteration on Gu * Gv (similar to a PSD matrix)
        for (int i = 0; i < r; ++i) v[i] = 1.0 + 0.01 * i;
        double lam = 0.0;
        for (int itn = 0; itn < 300; ++itn) {
          for (int i = 0; i < r; ++i) {
            double a = 0.0;
            for (int k = 0; k < r; ++k) a += Gv[i + (size_t)k * r] * v[k];
            z[i] = a;
          }
          double nrm = 0.0;
          for (int i = 0; i < r; ++i) {
            double a = 0.0;
            for (int k = 0; k < r; ++k) a += Gu[i + (size_t)k * r] * z[k];
            w[i] = a;
            nrm += a * a;
          }
          nrm = std::sqrt(nrm);
          double vn = 0.0;
          for (int i = 0; i < r; ++i) vn += v[i] * v[i];
          lam = nrm / std::sqrt(vn);
          if (nrm == 0.0) break;
          for (int i = 0; i < r; ++i) v[i] = w[i] / nrm;
        }
        const double norm = std::sqrt(lam);
        const double f = norm > 0.0 ? std::sqrt(offdiag_norm / norm) : 1.0;
        scale_u[c] = f;   // U_c and V_sb both take the factor
        scale_v[sb] = f;
      }
    }
    DevBuf<double> fac;
    std::vector<double> hf;
    for (size_t i = 1; i < t.nodes.size(); ++i) { hf.push_back(scale_u[i]); hf.push_back(scale_v[i]); }
    fac.upload(hf);
    std::vector<FillTask> sc;
    long long smax = 0;
    for (size_t i = 1; i < t.nodes.size(); ++i) {
      const Node &c = t.nodes[i];
      FillTask f{};
      f.lda = N;
      f.rows = c.nrow;
      f.a = S.U.p + c.row_beg + (long long)(c.col_beg - m) * N;
      f.cols = c.ncol;
      f.factor = fac.p + 2 * (i - 1);
      sc.push_back(f);
      f.a = S.V.p + c.row_beg + (long long)(c.col_beg - m) * N;
      f.cols = c.vncol;
      f.factor = fac.p + 2 * (i - 1) + 1;
      sc.push_back(f);
      smax = std::max(smax, (long long)c.nrow * std::max(c.ncol, c.vncol));
    }
    DevBuf<FillTask> dsc;
    dsc.upload(sc);
    launch_scale_batched(dsc.p, (int)sc.size(), smax, s);
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    S.factored = -1;
    return 0;
  });
}

int hodlr_set_leaf_size(hodlr_system h, int leaf_size) {
  if (!h) return -1;
  if (leaf_size < 1) return -2;
  System &S = h->sys;
  if (leaf_size > 1 && 2 * S.r > kMaxNodeS) return HODLR_ERR_UNSUPPORTED;
  if (leaf_size == S.leaf_size) return 0;
  return guarded([&]() -> int {
    S.leaf_size = leaf_size;
    S.fused64[0].built = S.fused64[1].built = false;
    S.reset_graphs();
    if (S.factored == HODLR_PREC_FP64) S.factored = -1;
    return 0;
  });
}

int hodlr_get_num_leaf(hodlr_system h) {
  if (!h) return -1;
  return (int)legion_leaves(h->sys.tree, h->sys.leaf_size).size();
}

int hodlr_legion_leaves(hodlr_system h, int *ids, int cap) {
  if (!h) return -1;
  const std::vector<int> v = legion_leaves(h->sys.tree, h->sys.leaf_size);
  if (ids) {
    if (cap < (int)v.size()) return -3;
    std::memcpy(ids, v.data(), sizeof(int) * v.size());
  }
  return (int)v.size();
}

int hodlr_solve_fused(hodlr_system h, int schur2, int sync, hodlr_stream_t stream) {
  if (!h) return -1;
  if (schur2 && 2 * h->sys.r > kMaxNodeS) return HODLR_ERR_UNSUPPORTED;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    System &S = h->sys;
    const int form = schur2 ? 1 : 0;
    S.ensure_fp64();
    S.run_graph(S.g_fused64[form], s, [&]() { S.run_fused64(form, s); });
    S.factored = HODLR_PREC_FP64;
    S.factored_form = form;
    if (sync) {
      const int info = S.check_info(s);
      if (int t = tc_status()) return t;
      return info;
    }
    return 0;
  });
}

int hodlr_factor(hodlr_system h, int precision, hodlr_stream_t stream) {
  if (!h) return -1;
  if (precision != HODLR_PREC_FP64 && precision != HODLR_PREC_MIXED) return -2;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    if (precision == HODLR_PREC_FP64) h->sys.run_fused64(0, s);
    else h->sys.run_factor32(s);
    const int info = h->sys.check_info(s);
    if (int t = tc_status()) return t;
    return info;
  });
}

int hodlr_solve(hodlr_system h, hodlr_stream_t stream) {
  if (!h) return -1;
  System &S = h->sys;
  if (S.factored < 0) return HODLR_ERR_STATE;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    const size_t nm = (size_t)S.N * S.m;
    if (S.factored == HODLR_PREC_FP64) {
      HODLR_CUDA_TRY(cudaMemcpyAsync(S.Y64.p, S.B.p, sizeof(double) * nm, cudaMemcpyDeviceToDevice, s));
      S.run_apply64(s);
      HODLR_CUDA_TRY(cudaMemcpyAsync(S.Xsol.p, S.Y64.p, sizeof(double) * nm, cudaMemcpyDeviceToDevice, s));
    } else {
      launch_convert2d<double, float>(S.B.p, S.N, S.Y32.p, S.N, S.N, S.m, s);
      S.run_apply32(s);
      launch_convert2d<float, double>(S.Y32.p, S.N, S.Xsol.p, S.N, S.N, S.m, s);
    }
    return 0;
  });
}

// The refined solve of one system on stream s (see hodlr_solve_refined).
// With `lane` (V still being copied in on lane->stream, lane->level_v[l]
// recorded once level l's columns of V are in, lane->v once all are), the
// mixed factor pass replays its leaf factorization, then runs the levels
// eagerly, each after its own columns of V arrived (converted to FP32 just
// before it), and the residual after all of V.
static int refined_body(System &S, int precision, double tol, int maxiter, int *iters,
                        double *relres, cudaStream_t s, const CopyLane *lane = nullptr) {
  const long long N = S.N;
  const size_t nm = (size_t)N * S.m;
  // two replayable segments: factor pass + residual, and one refinement
  // sweep + residual (captured as CUDA graphs on the first call)
  if (precision == HODLR_PREC_MIXED && lane) {
    S.ensure_mixed();
    S.run_graph(S.g_factor32_leaves, s, [&]() { S.run_factor32_part(kPathLeaves, s); });
    const LevelHook hook = [&](int l, int lo, int hi) {
      HODLR_CUDA_TRY(cudaStreamWaitEvent(s, lane->level_v[l], 0));
      S.convert_v32(lo, hi, s);
    };
    S.run_factor32_levels_hooked(hook, s);
    HODLR_CUDA_TRY(cudaStreamWaitEvent(s, lane->v, 0));  // the residual reads all of V
    launch_convert2d<float, double>(S.X32.p, N, S.Xsol.p, N, N, S.m, s);
    S.relres_enqueue(s);
    S.factored = HODLR_PREC_MIXED;
    S.factored_form = 0;
  } else if (precision == HODLR_PREC_MIXED) {
    S.ensure_mixed();
    S.run_graph(S.g_factor32, s, [&]() {
      S.run_factor32(s);
      launch_convert2d<float, double>(S.X32.p, N, S.Xsol.p, N, N, S.m, s);
      S.relres_enqueue(s);
    });
    S.factored = HODLR_PREC_MIXED;  // (host state is not part of a replay)
    S.factored_form = 0;
  } else {
    S.ensure_fp64();
    S.run_graph(S.g_factor64, s, [&]() {
      S.run_fused64(0, s);
      S.relres_enqueue(s);
    });
    S.factored = HODLR_PREC_FP64;
    S.factored_form = 0;
  }
  int info = S.check_info(s);
  // a factor pass whose engine gave up is wrong: report that, not its INFO
  if (int t = tc_status()) return t;
  if (info) return info;
  int it = 0;
  double rr = S.relres_read(s);
  while (rr > tol && it < maxiter) {
    if (precision == HODLR_PREC_MIXED) {
      S.run_graph(S.g_sweep32, s, [&]() {
        launch_convert2d<double, float>(S.R64.p, N, S.Y32.p, N, N, S.m, s);
        S.run_apply32(s);
        launch_add2d<float>(S.Xsol.p, N, S.Y32.p, N, N, S.m, s);
        S.relres_enqueue(s);
      });
    } else {
      S.run_graph(S.g_sweep64, s, [&]() {
        HODLR_CUDA_TRY(cudaMemcpyAsync(S.Y64.p, S.R64.p, sizeof(double) * nm,
                                       cudaMemcpyDeviceToDevice, s));
        S.run_apply64(s);
        launch_add2d<double>(S.Xsol.p, N, S.Y64.p, N, N, S.m, s);
        S.relres_enqueue(s);
      });
    }
    ++it;
    rr = S.relres_read(s);
  }
  if (iters) *iters = it;
  if (relres) *relres = rr;
  if (int t = tc_status()) return t;
  return rr <= tol ? 0 : HODLR_ERR_NOCONV;
}

int hodlr_solve_refined(hodlr_system h, int precision, double tol, int maxiter, int *iters,
                        double *relres, hodlr_stream_t stream) {
  if (!h) return -1;
  if (precision != HODLR_PREC_FP64 && precision != HODLR_PREC_MIXED) return -2;
  if (!(tol >= 0.0)) return -3;
  if (maxiter < 0) return -4;
  return guarded([&]() -> int {
    return refined_body(h->sys, precision, tol, maxiter, iters, relres, as_stream(stream));
  });
}

int hodlr_solve_refined_host(hodlr_system h, const double *D, long long ldd, const double *U,
                             long long ldu, const double *V, long long ldv, const double *B,
                             long long ldb, double *X, long long ldx, int precision, double tol,
                             int maxiter, int *iters, double *relres, hodlr_stream_t stream) {
  if (!h) return -1;
  System &S = h->sys;
  if (!D) return -2;
  if (ldd < S.N) return -3;
  if (S.vc > 0 && !U) return -4;
  if (S.vc > 0 && ldu < S.N) return -5;
  if (S.vc > 0 && !V) return -6;
  if (S.vc > 0 && ldv < S.N) return -7;
  if (!B) return -8;
  if (ldb < S.N) return -9;
  if (!X) return -10;
  if (ldx < S.N) return -11;
  if (precision != HODLR_PREC_FP64 && precision != HODLR_PREC_MIXED) return -12;
  if (!(tol >= 0.0)) return -13;
  if (maxiter < 0) return -14;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    // no return while a copy may still read the caller's buffers
    struct DrainLane {
      cudaStream_t st = nullptr;
      ~DrainLane() {
        if (st) cudaStreamSynchronize(st);
      }
    } drain;
    copy2d(S.D.p, S.N, D, ldd, S.N, S.nmax, 1, s);
    copy2d(S.B.p, S.N, B, ldb, S.N, S.m, 1, s);
    if (S.vc > 0) copy2d(S.U.p, S.N, U, ldu, S.N, S.vc, 1, s);
    S.factored = -1;
    const CopyLane *lane = nullptr;
    if (S.vc > 0 && precision == HODLR_PREC_MIXED) {
      // V is first read by the tree levels, each level only its children's
      // columns: V follows the other copies on the copy lane, in the levels'
      // order (deepest first), one event per level, under the leaf
      // factorization and the levels before
      S.ensure_mixed();
      const auto &lv = S.fused32.levels;
      S.lane.ensure();
      S.lane.ensure_levels(lv.size());
      drain.st = S.lane.stream;
      HODLR_CUDA_TRY(cudaEventRecord(S.lane.inputs, s));
      HODLR_CUDA_TRY(cudaStreamWaitEvent(S.lane.stream, S.lane.inputs, 0));
      int covered = S.vc;  // columns [covered, vc) of V are on their way
      for (size_t l = 0; l < lv.size(); ++l) {
        const int lo = lv[l]->v_hi > lv[l]->v_lo ? std::min(lv[l]->v_lo, covered) : covered;
        if (lo < covered) {
          copy2d(S.V.p + (size_t)lo * S.N, S.N, V + (size_t)lo * ldv, ldv, S.N, covered - lo, 1,
                 S.lane.stream);
          covered = lo;
        }
        HODLR_CUDA_TRY(cudaEventRecord(S.lane.level_v[l], S.lane.stream));
      }
      if (covered > 0) copy2d(S.V.p, S.N, V, ldv, S.N, covered, 1, S.lane.stream);
      HODLR_CUDA_TRY(cudaEventRecord(S.lane.v, S.lane.stream));
      lane = &S.lane;
    } else if (S.vc > 0) {
      copy2d(S.V.p, S.N, V, ldv, S.N, S.vc, 1, s);
    }
    const int rc = refined_body(S, precision, tol, maxiter, iters, relres, s, lane);
    HODLR_CUDA_TRY(cudaMemcpy2DAsync(X, sizeof(double) * ldx, S.Xsol.p, sizeof(double) * S.N,
                                     sizeof(double) * S.N, S.m, cudaMemcpyDeviceToHost, s));
    HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return rc;
  });
}

// ---------------------------------------------------------------------------
// launch schedule and its autotuner
// ---------------------------------------------------------------------------

static hodlr_schedule schedule_of(const System &S) {
  hodlr_schedule c{};
  c.leaf_nb = S.nb32;
  c.leaf_ob32 = S.ob32;
  c.leaf_ob64 = S.ob64;
  c.reduce_rows = S.red_chunk;
  c.bcast_rows = S.bc_chunk;
  return c;
}

// 0, or the negative index of the first invalid field (as an argument error)
static int schedule_check(const System &S, const hodlr_schedule &c) {
  if (c.leaf_nb != 0 && c.leaf_nb != 32 && c.leaf_nb != 64) return -2;
  if (c.leaf_nb == 64 && S.nmax > 512) return -2;  // the 64-wide panel holds <= 512 rows
  if (c.leaf_ob32 < 0 || c.leaf_ob32 > 1024) return -3;
  if (c.leaf_ob64 < 0 || c.leaf_ob64 > 1024) return -4;
  if (c.reduce_rows < 16 || c.reduce_rows > 65536 || c.reduce_rows % 16) return -5;
  if (c.bcast_rows < 16 || c.bcast_rows > 65536 || c.bcast_rows % 16) return -6;
  return 0;
}

// Installs a (checked) schedule: the launch plans and captured graphs are
// rebuilt on the next solve, and the system must be factored again.
static void schedule_apply(System &S, const hodlr_schedule &c) {
  const hodlr_schedule cur = schedule_of(S);
  if (std::memcmp(&cur, &c, sizeof(c)) == 0) return;
  S.nb32 = c.leaf_nb;
  S.ob32 = c.leaf_ob32;
  S.ob64 = c.leaf_ob64;
  S.red_chunk = c.reduce_rows;
  S.bc_chunk = c.bcast_rows;
  S.fused32.built = false;
  S.fused64[0].built = S.fused64[1].built = false;
  S.reset_graphs();
  S.factored = -1;
}

int hodlr_get_schedule(hodlr_system h, hodlr_schedule *out) {
  if (!h) return -1;
  if (!out) return -2;
  *out = schedule_of(h->sys);
  return 0;
}

int hodlr_set_schedule(hodlr_system h, const hodlr_schedule *in) {
  if (!h) return -1;
  if (!in) return -2;
  if (int rc = schedule_check(h->sys, *in)) return rc;
  return guarded([&]() -> int {
    schedule_apply(h->sys, *in);
    return 0;
  });
}

}  // extern "C"

namespace {

// Coordinate search over the schedule fields: each field in turn takes the
// candidate value with the smallest measured time (the others fixed), until a
// full pass changes nothing (at most `passes` passes).  `measure` installs a
// schedule, runs the timed solves and returns the mean milliseconds (< 0 if
// the schedule failed).
template <typename M>
int tune_search(hodlr_schedule &best, double &best_ms, int precision,
                const std::vector<int> &nb_opts, M &&measure, hodlr_tune_trial *log, int log_cap,
                int *n_log) {
  int nlog = 0;
  auto record = [&](const hodlr_schedule &c, double ms) {
    if (log && nlog < log_cap) log[nlog] = hodlr_tune_trial{c, ms};
    ++nlog;
  };
  best_ms = measure(best);
  record(best, best_ms);
  if (!(best_ms >= 0)) return HODLR_ERR_CUDA;
  const std::vector<int> rows = {256, 512, 1024, 2048};
  const std::vector<int> ob32 = {0, 128, 256};
  const std::vector<int> ob64 = {0, 64, 128};
  const int nfields = 4;
  for (int pass = 0; pass < 2; ++pass) {
    bool changed = false;
    for (int f = 0; f < nfields; ++f) {
      std::vector<int> opts;
      if (f == 0) opts = precision == HODLR_PREC_MIXED ? ob32 : ob64;
      else if (f == 1) opts = precision == HODLR_PREC_MIXED ? nb_opts : std::vector<int>{};
      else opts = rows;
      for (int v : opts) {
        hodlr_schedule c = best;
        int &field = f == 0 ? (precision == HODLR_PREC_MIXED ? c.leaf_ob32 : c.leaf_ob64)
                     : f == 1 ? c.leaf_nb
                     : f == 2 ? c.reduce_rows
                              : c.bcast_rows;
        if (field == v) continue;
        field = v;
        const double ms = measure(c);
        record(c, ms);
        if (ms >= 0 && ms < 0.98 * best_ms) {  // keep a change only for a clear gain
          best = c;
          best_ms = ms;
          changed = true;
        }
      }
    }
    if (!changed) break;
  }
  if (n_log) *n_log = nlog;
  return 0;
}

// mean milliseconds of `reps` calls of fn on stream s (after one untimed call)
template <typename F>
double time_calls(cudaStream_t s, int reps, F &&fn) {
  if (fn() < 0) return -1.0;
  cudaEvent_t e0, e1;
  HODLR_CUDA_TRY(cudaEventCreate(&e0));
  HODLR_CUDA_TRY(cudaEventCreate(&e1));
  HODLR_CUDA_TRY(cudaEventRecord(e0, s));
  int rc = 0;
  for (int i = 0; i < reps && rc >= 0; ++i) rc = fn();
  HODLR_CUDA_TRY(cudaEventRecord(e1, s));
  HODLR_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc < 0 ? -1.0 : (double)ms / reps;
}

std::vector<int> nb_options(int nmax) {
  std::vector<int> v = {0};
  if (nmax <= 512) v.push_back(32);  // the default is 64 there
  return v;
}

// A private stream for tuning: the solves are captured as CUDA graphs only
// on a non-default stream, and the timed configuration is the replayed one.
struct TuneStream {
  cudaStream_t s = nullptr;
  TuneStream() {
    HODLR_CUDA_TRY(cudaDeviceSynchronize());
    HODLR_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  }
  ~TuneStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

}  // namespace

extern "C" {

int hodlr_autotune(hodlr_system h, int precision, double tol, int reps, hodlr_schedule *best,
                   double *best_ms, hodlr_tune_trial *log, int log_cap, int *n_log) {
  if (!h) return -1;
  if (precision != HODLR_PREC_FP64 && precision != HODLR_PREC_MIXED) return -2;
  if (!(tol >= 0.0)) return -3;
  if (reps < 1) return -4;
  if (log_cap < 0) return -7;
  return guarded([&]() -> int {
    System &S = h->sys;
    TuneStream ts;
    auto measure = [&](const hodlr_schedule &c) -> double {
      if (schedule_check(S, c)) return -1.0;
      schedule_apply(S, c);
      return time_calls(ts.s, reps, [&]() -> int {
        if (precision == HODLR_PREC_MIXED)
          return refined_body(S, precision, tol, 10, nullptr, nullptr, ts.s);
        S.ensure_fp64();
        S.run_graph(S.g_fused64[0], ts.s, [&]() { S.run_fused64(0, ts.s); });
        S.factored = HODLR_PREC_FP64;
        S.factored_form = 0;
        return S.check_info(ts.s) ? -1 : 0;
      });
    };
    hodlr_schedule b = schedule_of(S);
    double ms = 0.0;
    int rc = tune_search(b, ms, precision, nb_options(S.nmax), measure, log, log_cap, n_log);
    if (rc) return rc;
    schedule_apply(S, b);
    if (best) *best = b;
    if (best_ms) *best_ms = ms;
    return 0;
  });
}

int hodlr_matvec(hodlr_system h, const double *x, long long ldx, double *y, long long ldy,
                 int ncols, hodlr_stream_t stream) {
  if (!h) return -1;
  System &S = h->sys;
  if (!x) return -2;
  if (ldx < S.N) return -3;
  if (!y) return -4;
  if (ldy < S.N) return -5;
  if (ncols < 0 || ncols > S.m) return -6;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    HODLR_CUDA_TRY(cudaMemsetAsync(S.MVx.p, 0, sizeof(double) * (size_t)S.N * S.m, s));
    copy2d(S.MVx.p, S.N, x, ldx, S.N, ncols, 0, s);
    S.run_matvec(S.mv_usr, 1.0, 0.0, s);
    copy2d(y, ldy, S.R64.p, S.N, S.N, ncols, 0, s);
    return 0;
  });
}

int hodlr_set_profiling(hodlr_system h, int on) {
  if (!h) return -1;
  return guarded([&]() -> int {
    h->sys.prof.reset();
    h->sys.prof.on = on != 0;
    return 0;
  });
}

static_assert(PH_COUNT == HODLR_PHASES, "phase list of the C ABI");

int hodlr_batch_create(hodlr_batch *out, const hodlr_system *systems, int count) {
  if (!out) return -1;
  *out = nullptr;
  if (!systems) return -2;
  if (count <= 0 || count > 16384) return -3;
  for (int k = 0; k < count; ++k)
    if (!systems[k]) return -2;
  if (int rc = device_ok()) return rc;
  return guarded([&]() -> int {
    auto *h = new hodlr_batch_s();
    try {
      std::vector<System *> v;
      for (int k = 0; k < count; ++k) v.push_back(&systems[k]->sys);
      h->b.build(v);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return 0;
  });
}

int hodlr_batch_destroy(hodlr_batch batch) {
  if (!batch) return -1;
  delete batch;
  return 0;
}

// The refined solve of every system of a batch on stream s.
static int batch_body(Batch &B, double tol, int maxiter, int *iters, double *relres_max,
                      double *relres, int *failed, cudaStream_t s) {
  B.run_graph(B.g_factor, s, [&]() { B.run_factor(s); });
  for (System *S : B.sys) {
    S->factored = HODLR_PREC_MIXED;
    S->factored_form = 0;
  }
  int info = B.check_info(s, failed);
  if (int t = tc_status()) return t;
  if (info) return info;
  std::vector<double> per;
  int it = 0;
  double rr = B.relres_read(s, &per);
  while (rr > tol && it < maxiter) {
    B.run_graph(B.g_sweep, s, [&]() { B.run_sweep(s); });
    ++it;
    rr = B.relres_read(s, &per);
  }
  if (int t = tc_status()) return t;
  if (iters) *iters = it;
  if (relres_max) *relres_max = rr;
  if (relres)
    for (size_t k = 0; k < per.size(); ++k) relres[k] = per[k];
  return rr <= tol ? 0 : HODLR_ERR_NOCONV;
}

int hodlr_batch_solve_refined(hodlr_batch batch, double tol, int maxiter, int *iters,
                              double *relres_max, double *relres, int *failed,
                              hodlr_stream_t stream) {
  if (!batch) return -1;
  if (!(tol >= 0.0)) return -2;
  if (maxiter < 0) return -3;
  return guarded([&]() -> int {
    return batch_body(batch->b, tol, maxiter, iters, relres_max, relres, failed,
                      as_stream(stream));
  });
}

int hodlr_batch_autotune(hodlr_batch batch, double tol, int reps, hodlr_schedule *best,
                         double *best_ms, hodlr_tune_trial *log, int log_cap, int *n_log) {
  if (!batch) return -1;
  if (!(tol >= 0.0)) return -2;
  if (reps < 1) return -3;
  if (log_cap < 0) return -6;
  return guarded([&]() -> int {
    Batch &B = batch->b;
    TuneStream ts;
    int nmax = 0;
    for (System *S : B.sys) nmax = std::max(nmax, S->nmax);
    auto measure = [&](const hodlr_schedule &c) -> double {
      for (System *S : B.sys)
        if (schedule_check(*S, c)) return -1.0;
      for (System *S : B.sys) schedule_apply(*S, c);
      B.build(B.sys);
      return time_calls(ts.s, reps, [&]() -> int {
        const int rc = batch_body(B, tol, 10, nullptr, nullptr, nullptr, nullptr, ts.s);
        return rc > 0 ? -1 : 0;
      });
    };
    hodlr_schedule b = schedule_of(*B.sys[0]);
    double ms = 0.0;
    int rc = tune_search(b, ms, HODLR_PREC_MIXED, nb_options(nmax), measure, log, log_cap, n_log);
    if (rc) return rc;
    for (System *S : B.sys) schedule_apply(*S, b);
    B.build(B.sys);
    if (best) *best = b;
    if (best_ms) *best_ms = ms;
    return 0;
  });
}

int hodlr_batch_set_profiling(hodlr_batch batch, int on) {
  if (!batch) return -1;
  return guarded([&]() -> int {
    batch->b.prof.reset();
    batch->b.prof.on = on != 0;
    return 0;
  });
}

int hodlr_batch_phase_times(hodlr_batch batch, double *ms, long long *launches, int reset) {
  if (!batch) return -1;
  return guarded([&]() -> int {
    Profiler &p = batch->b.prof;
    p.collect();
    for (int i = 0; i < PH_COUNT; ++i) {
      if (ms) ms[i] = p.ms[i];
      if (launches) launches[i] = p.launches[i];
    }
    if (reset) p.reset();
    return 0;
  });
}

int hodlr_phase_times(hodlr_system h, double *ms, long long *launches, int reset) {
  if (!h) return -1;
  return guarded([&]() -> int {
    Profiler &p = h->sys.prof;
    p.collect();
    for (int i = 0; i < PH_COUNT; ++i) {
      if (ms) ms[i] = p.ms[i];
      if (launches) launches[i] = p.launches[i];
    }
    if (reset) p.reset();
    return 0;
  });
}

int hodlr_relres(hodlr_system h, double *relres, hodlr_stream_t stream) {
  if (!h) return -1;
  if (!relres) return -2;
  return guarded([&]() -> int {
    *relres = h->sys.relres(as_stream(stream));
    return 0;
  });
}

int hodlr_get_solution(hodlr_system h, double *X, long long ldx, int host,
                       hodlr_stream_t stream) {
  if (!h) return -1;
  System &S = h->sys;
  if (!X) return -2;
  if (ldx < S.N) return -3;
  return guarded([&]() -> int {
    cudaStream_t s = as_stream(stream);
    HODLR_CUDA_TRY(cudaMemcpy2DAsync(X, sizeof(double) * ldx, S.Xsol.p, sizeof(double) * S.N,
                                     sizeof(double) * S.N, S.m,
                                     host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    if (host) HODLR_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  });
}

}  // extern "C"
