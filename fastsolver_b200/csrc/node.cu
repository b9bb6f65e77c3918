// node.cu -- capacitance (node) factorization, FP64, batched over a tree level.
//
// GPU restatement of LUSolveTask::cpu_task (src/solver/solver_tasks.cc:
// 139-305) and of the 2r x 2r Schur system of serial_leaf_solve's internal
// branch (solver_tasks.cc:483-535).  For a node with children b0, b1 and the
// summed reduce results W0 = [V0Td0 | V0Tu0], W1 = [V1Td1 | V1Tu1] the
// reference computes, per column block of the d part,
//
//   T    = V1Td1 - V1Tu1 V0Td0          (dgemm at 236)
//   eta0 = S^{-1} T,  S = I - V1Tu1 V0Tu0   (dgemm at 261, dgesv at 281)
//   eta1 = V0Td0 - V0Tu0 eta0           (dgemm at 299)
//
// which is linear in [V0Td0; V1Td1]:
//
//   [eta0; eta1] = M [V0Td0; V1Td1],
//   M = [[ -S^{-1} V1Tu1,            S^{-1}         ],
//        [ I + V0Tu0 S^{-1} V1Tu1,  -V0Tu0 S^{-1}   ]]
//
// (form 1, the 2r x 2r system [[V0Tu0, I], [I, V1Tu1]] of the leaf-internal
// branch: M is that matrix's inverse).  node_factor_kernel forms M once per
// node -- one CTA per node, S^{-1} by Gauss-Jordan elimination with partial
// pivoting (pivot = largest |a|, lowest row on ties, as LAPACK's idamax; in
// registers for s <= 64, in shared memory above), the three products from
// shared memory and L2 (and S itself where V0Tu0, V1Tu1 fit in shared
// memory) -- and the
// solver applies M to every column block as one batched GEMM per level (the
// same engine as the reduce and broadcast), for the fused pass and for every
// later solve with the same factors.  INFO > 0 reports an exactly zero pivot
// (singular S), as dgesv.
#include <algorithm>

#include "common.cuh"
#include "node.cuh"

namespace hodlr {

namespace {

constexpr int kNodeThreads = 512;
constexpr int kNodeWarps = kNodeThreads / 32;
// published candidate rows of the register elimination: [2][kNodeWarps][64]
constexpr size_t kGjScratchWords = 2 * kNodeWarps * 64;

}  // namespace

// doubles of the factor kernel's shared memory before the staged operands:
// A (s x (s + 1)), rowk, colk (s each), piv, src, at (s ints each), rounded up
__host__ __device__ size_t node_factor_words(int max_s) {
  return (size_t)max_s * (max_s + 1) + 2 * (size_t)max_s + 2 * (size_t)max_s + 2;
}

namespace {

// Warp-wide argmax of |a| (>= 0, so its bit pattern orders like the value)
// with the lowest position on ties; lanes without a candidate pass
// pos = INT_MAX.  Every lane gets the winner's (best, pos, code); pos stays
// INT_MAX (code -1) when no lane had a candidate.
__device__ inline void warp_argmax_f64(double &best, int &pos, int &code, int &wlane) {
  const bool cand = pos != 0x7fffffff;
  const unsigned long long b = cand ? (unsigned long long)__double_as_longlong(best) : 0ull;
  const unsigned hi = (unsigned)(b >> 32), lo = (unsigned)b;
  const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
  const bool top = hi == mh && lo == ml;
  const unsigned pm = __reduce_min_sync(0xffffffffu, top ? (unsigned)pos : 0xffffffffu);
  const unsigned win = __ballot_sync(0xffffffffu, cand && top && (unsigned)pos == pm);
  wlane = win ? __ffs(win) - 1 : 0;
  best = __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
  pos = win ? (int)pm : 0x7fffffff;
  code = __shfl_sync(0xffffffffu, code, wlane);
  if (!win) code = -1;
}

// out(i, c) = [i == c] (if add_identity) + alpha * sum_k a(i, k) b(k, c) for
// i < rows, c < cols: lanes over rows, warps over columns, 2 x 2 outputs per
// thread and pass.
template <typename FA, typename FB, typename FO>
__device__ inline void node_product(int rows, int cols, int K, double alpha, bool add_identity,
                                    FA a, FB b, FO out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = lane; i0 < rows; i0 += 64) {
    const int i1 = i0 + 32 < rows ? i0 + 32 : i0;
    for (int c0 = warp; c0 < cols; c0 += 2 * kNodeWarps) {
      const int c1 = c0 + kNodeWarps < cols ? c0 + kNodeWarps : c0;
      double a00 = 0.0, a01 = 0.0, a10 = 0.0, a11 = 0.0;
#pragma unroll 8
      for (int k = 0; k < K; ++k) {
        const double x0 = a(i0, k), x1 = a(i1, k);
        const double y0 = b(k, c0), y1 = b(k, c1);
        a00 += x0 * y0;
        a01 += x0 * y1;
        a10 += x1 * y0;
        a11 += x1 * y1;
      }
      auto put = [&](int i, int c, double v) {
        out(i, c, (add_identity && i == c ? 1.0 : 0.0) + alpha * v);
      };
      put(i0, c0, a00);
      if (c1 != c0) put(i0, c1, a01);
      if (i1 != i0) {
        put(i1, c0, a10);
        if (c1 != c0) put(i1, c1, a11);
      }
    }
  }
}

// The same product with both operands FP64 column-major in shared memory,
// on the FP64 tensor pipe (mma.m16n8k4.f64): every warp takes 16 x 8 output
// tiles in turn.  Fragments (g = lane / 4, t = lane % 4): A a0 = A[g][t],
// a1 = A[g + 8][t]; B b = B[t][g]; C c0..c3 = C[g][2t], C[g][2t + 1],
// C[g + 8][2t], C[g + 8][2t + 1].  Against the SIMT product it reads a
// fifth of the shared-memory bytes per multiply-add.  FP32 operands (the
// mixed path's staged V^T u blocks) convert to FP64 exactly at the load.
template <typename TA, typename TB, typename FO>
__device__ inline void node_product_dmma(int rows, int cols, int K, double alpha,
                                         bool add_identity, const TA *A, int lda, const TB *B,
                                         int ldb, FO out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int tm = (rows + 15) / 16, tn = (cols + 7) / 8;
  for (int tile = warp; tile < tm * tn; tile += kNodeWarps) {
    const int m0 = (tile / tn) * 16, n0 = (tile % tn) * 8;
    double c[4] = {0.0, 0.0, 0.0, 0.0};
    const int ra = m0 + g, rb = m0 + g + 8, cb = n0 + g;
    for (int k = 0; k < K; k += 4) {
      const int kk = k + t;
      const bool kin = kk < K;
      const double a0 = (kin && ra < rows) ? double(A[ra + kk * lda]) : 0.0;
      const double a1 = (kin && rb < rows) ? double(A[rb + kk * lda]) : 0.0;
      const double b = (kin && cb < cols) ? double(B[kk + cb * ldb]) : 0.0;
      asm volatile(
          "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
          "{%0, %1, %2, %3};\n"
          : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
          : "d"(a0), "d"(a1), "d"(b));
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = m0 + g + (v >> 1) * 8, j = n0 + 2 * t + (v & 1);
      if (i < rows && j < cols) out(i, j, (add_identity && i == j ? 1.0 : 0.0) + alpha * c[v]);
    }
  }
}

// Gauss-Jordan elimination with implicit row interchanges of the s x s
// matrix A (s <= 64, row-major in shared memory, row stride lda), the same
// steps as the shared-memory elimination of node_factor_kernel but on
// registers: warp w holds rows 4w .. 4w + 3, lane (row, g) (g = lane % 8)
// columns g, g + 8, ..., g + 56 of its row.  Per column k every warp finds
// its best candidate (largest |a| among the rows not yet pivotal, lowest
// current position on ties, as idamax after LAPACK's interchanges) and the
// candidate row's 8 lanes publish the row (double-buffered); one barrier;
// every warp combines the 16 candidates and eliminates column k from its rows
// with the published (unscaled) pivot row, while the pivot row's lanes scale
// their own values.  Measured on B200 with s = 64: the shared-memory form
// spent ~3.5 k cycles per column, mostly re-reading and re-writing the whole
// matrix in shared memory.  On return A holds the eliminated matrix (the
// input of the inverse's gather), piv[k] the interchange of step k, at[i] the
// storage row at final position i, *s_info the first zero pivot (1-based) or
// 0.  scratch: kGjScratchWords doubles of shared memory for the published
// candidate rows (the caller's, so that it can share them with buffers that
// are dead during the elimination).  Every thread of the CTA calls it.
__device__ inline void gj_registers(double *A, int lda, int s, int *piv, int *at, int *s_info,
                                    double *scratch) {
  constexpr int NWG = kNodeWarps;
  auto wrow = reinterpret_cast<double (*)[NWG][64]>(scratch);  // [2][NWG][64]
  __shared__ double wval[2][NWG];
  __shared__ int wpos[2][NWG], wcode[2][NWG];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i = 4 * warp + (lane >> 3);  // this lane's row
  const int g = lane & 7;                // its column group
  const bool rowok = i < s;
  double a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = g + 8 * j;
    a[j] = (rowok && c < s) ? A[i * lda + c] : 0.0;
  }
  int pos = i;          // current position of row i (LAPACK interchange order)
  bool used = !rowok;   // row already pivotal (or absent)
  int info = 0;
  for (int k = 0; k < s; ++k) {
    const int slot = k & 1, kg = k & 7, kj = k >> 3;
    // A[i][k], held by lane (row, kg) at register kj
    double mine = a[0];
#pragma unroll
    for (int j = 1; j < 8; ++j)
      if (j == kj) mine = a[j];
    const double aik = __shfl_sync(0xffffffffu, mine, (lane & ~7) | kg);
    double best = 0.0;
    int bp = 0x7fffffff, code = -1;
    if (g == kg && !used) {
      const double av = fabs(aik);
      if (av == av) { best = av; bp = pos; code = i; }  // NaN is never a candidate
    }
    int wl;
    warp_argmax_f64(best, bp, code, wl);
    if (code >= 0 && i == code) {  // the warp's candidate row publishes itself
#pragma unroll
      for (int j = 0; j < 8; ++j) wrow[slot][warp][g + 8 * j] = a[j];
    }
    if (lane == 0) { wval[slot][warp] = best; wpos[slot][warp] = bp; wcode[slot][warp] = code; }
    __syncthreads();
    double pb = 0.0;
    int pp = 0x7fffffff, pc = -1, pw = 0;
    if (lane < NWG) { pb = wval[slot][lane]; pp = wpos[slot][lane]; pc = wcode[slot][lane]; }
    warp_argmax_f64(pb, pp, pc, pw);  // pw: the winning warp
    const double pk = pc >= 0 ? wrow[slot][pw][k] : 0.0;
    if (pk == 0.0) {  // exactly singular (or a NaN column): INFO = k + 1, uniform
      info = k + 1;
      break;
    }
    if (tid == 0) piv[k] = pp;
    const double rinv = 1.0 / pk;
    if (rowok) {
      if (i == pc) {
        pos = k;
        used = true;
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = (g + 8 * j == k) ? rinv : a[j] * rinv;
      } else {
        if (pos == k) pos = pp;
        const double f = aik * rinv;
        const double *prow = wrow[slot][pw];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int c = g + 8 * j;
          a[j] = (c == k) ? -f : a[j] - f * prow[c];
        }
      }
    }
  }
  if (rowok) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = g + 8 * j;
      if (c < s) A[i * lda + c] = a[j];
    }
    if (g == 0 && info == 0) at[pos] = i;
  }
  if (tid == 0) *s_info = info;
}

template <typename TW, typename TE, int RL>
__global__ void __launch_bounds__(kNodeThreads)
    node_factor_kernel(const NodeTask<TW, TE> *tasks, int form, int max_s, int max_r, int stage,
                       int galias, int *info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const NodeTask<TW, TE> tk = tasks[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = tk.r0, r1 = tk.r1, s2 = r0 + r1;
  const int s = form == 0 ? r0 : s2;
  const int lda = s + 1;                              // row stride (odd: no bank conflicts)
  double *A = reinterpret_cast<double *>(smem_raw);   // s x s, row-major
  // two s-double slots after A are spare; the int arrays follow them
  int *piv = reinterpret_cast<int *>(A + (size_t)s * lda + 2 * s);
  int *src = piv + s;
  int *at = src + s;
  // form 0 with stage != 0: V0Tu0 and V1Tu1 in shared memory in their own
  // precision (the products convert them), then S^{-1} un-permuted and
  // G0 = -S^{-1} V1Tu1, both FP64 column-major.  With galias (r1 <= r0 + 1
  // for every node of the launch) G0 takes the eliminated matrix's place,
  // which is dead once S^{-1} has been gathered.
  // The register elimination's candidate-row scratch shares the S^{-1} / G0
  // region (both are written after the elimination).
  TW *W0s = reinterpret_cast<TW *>(reinterpret_cast<double *>(smem_raw) + node_factor_words(max_s));
  TW *W1s = W0s + (stage ? (size_t)max_r * max_r : 0);
  double *Ts = reinterpret_cast<double *>(W1s + (stage ? (size_t)max_r * max_r : 0));
  double *Ss = Ts;
  double *Gs = galias ? A : Ss + (size_t)max_r * max_r;
  __shared__ int s_info;

  if (tid == 0) s_info = 0;
  if (form == 0 && stage) {
    for (int e = tid; e < r1 * r0; e += kNodeThreads) {
      const int i = e % r1, j = e / r1;
      W0s[e] = tk.W0u[i + (long long)j * tk.ldw0u];
    }
    for (int e = tid; e < r0 * r1; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      W1s[e] = tk.W1u[i + (long long)j * tk.ldw1u];
    }
  }
  if (form == 0 && stage) {
    // S = I - V1Tu1 V0Tu0 (the dgemm at solver_tasks.cc:261) from the staged
    // FP64 copies, on the DMMA pipe, straight into the elimination's matrix
    __syncthreads();
    node_product_dmma(r0, r0, r1, -1.0, true, W1s, r0, W0s, r1,
                      [&](int i, int c, double v) { A[i * lda + c] = v; });
  } else if (form == 0) {
    for (int e = tid; e < s * s; e += kNodeThreads) {
      const int i = e % s, c = e / s;
      A[i * lda + c] = tk.S[e];
    }
  } else {
    for (int e = tid; e < s * s; e += kNodeThreads) {
      const int i = e % s, c = e / s;
      double v = (i == (r1 + c) % s) ? 1.0 : 0.0;
      if (i < r1 && c < r0) v = double(tk.W0u[i + (long long)c * tk.ldw0u]);
      else if (i >= r1 && c >= r0) v = double(tk.W1u[(i - r1) + (long long)(c - r0) * tk.ldw1u]);
      A[i * lda + c] = v;
    }
  }
  __syncthreads();

  if constexpr (RL <= 2) {
    gj_registers(A, lda, s, piv, at, &s_info, Ts);
  } else {
    // ---- Gauss-Jordan with implicit row interchanges, one barrier per column.
    // Rows never move; every warp finds the pivot of column k itself (largest
    // |a| among the rows not yet pivotal, lowest current position on ties, as
    // idamax after LAPACK's interchanges) and keeps identical copies of the
    // rows' current positions.  Warp w eliminates column k from rows w, w + kNodeWarps,
    // ... with the (unscaled) pivot row; the pivot row itself is scaled by its
    // owner at the start of the next step, when nobody else reads it.
    // RL: rows (and columns) per lane, ceil(max_s / 32)
    int posr[RL];
    bool usedr[RL];
  #pragma unroll
    for (int t = 0; t < RL; ++t) {
      const int row = lane + 32 * t;
      posr[t] = row;
      usedr[t] = row >= s;
    }
    int prevp = -1, prevk = -1;
    double prevr = 0.0;
    auto scale_prev = [&]() {
      if (prevp >= 0 && (prevp % kNodeWarps) == warp) {
        double *Ap = A + prevp * lda;
        for (int c = lane; c < s; c += 32) Ap[c] = (c == prevk) ? prevr : Ap[c] * prevr;
      }
    };
    for (int k = 0; k < s; ++k) {
      scale_prev();
      // the owner warp's lanes wrote the previous pivot row, whose column k the
      // same warp reads below (Ai[k] of its rows): order those accesses
      __syncwarp();
      double best = 0.0;
      int bp = 0x7fffffff, code = -1;
  #pragma unroll
      for (int t = 0; t < RL; ++t) {
        const int row = lane + 32 * t;
        if (row < s && !usedr[t]) {
          const double av = fabs(A[row * lda + k]);
          if (av == av && (bp == 0x7fffffff || av > best || (av == best && posr[t] < bp))) {
            best = av; bp = posr[t]; code = row;
          }
        }
      }
      int wl;
      warp_argmax_f64(best, bp, code, wl);
      const int p = code, pp = bp;
      const double pk = p >= 0 ? A[p * lda + k] : 0.0;
      if (pk == 0.0) {  // exactly singular (or a NaN column): INFO = k + 1, uniform
        if (tid == 0) s_info = k + 1;
        break;
      }
  #pragma unroll
      for (int t = 0; t < RL; ++t) {
        const int row = lane + 32 * t;
        if (row == p) { posr[t] = k; usedr[t] = true; }
        else if (posr[t] == k) posr[t] = pp;
      }
      if (tid == 0) piv[k] = pp;
      const double rinv = 1.0 / pk;
      double prow[RL];
  #pragma unroll
      for (int u = 0; u < RL; ++u) {
        const int c = lane + 32 * u;
        prow[u] = c < s ? A[p * lda + c] : 0.0;
      }
      // this warp's rows i = warp, warp + kNodeWarps, ...: all multipliers are
      // read before any lane writes column k (one __syncwarp), so the row
      // updates are independent and overlap
      constexpr int RW = (kMaxNodeS + kNodeWarps - 1) / kNodeWarps;
      double fr[RW];
  #pragma unroll
      for (int jj = 0; jj < RW; ++jj) {
        const int i = warp + kNodeWarps * jj;
        fr[jj] = (i < s && i != p) ? A[i * lda + k] * rinv : 0.0;
      }
      __syncwarp();
  #pragma unroll
      for (int jj = 0; jj < RW; ++jj) {
        const int i = warp + kNodeWarps * jj;
        if (i >= s || i == p) continue;
        double *Ai = A + i * lda;
  #pragma unroll
        for (int u = 0; u < RL; ++u) {
          const int c = lane + 32 * u;
          if (c < s) Ai[c] = (c == k) ? -fr[jj] : Ai[c] - fr[jj] * prow[u];
        }
      }
      prevp = p;
      prevk = k;
      prevr = rinv;
      __syncthreads();
    }
    __syncthreads();  // s_info (set on the singular break) visible to all
    if (s_info == 0) scale_prev();
    // at[i]: the storage row at final position i (every warp holds the same posr)
    if (warp == 0) {
  #pragma unroll
      for (int t = 0; t < RL; ++t) {
        const int row = lane + 32 * t;
        if (row < s) at[posr[t]] = row;
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (info) info[tk.info_slot] = s_info;
    // undo the row interchanges as column interchanges, last pivot first
    for (int j = 0; j < s; ++j) src[j] = j;
    if (s_info == 0)
      for (int k = s - 1; k >= 0; --k) {
        const int p = piv[k];
        const int t = src[k];
        src[k] = src[p];
        src[p] = t;
      }
  }
  __syncthreads();
  if (s_info != 0) return;  // singular: no solve matrix (uniform across the CTA)
  // S^{-1}(i, j) = A[at[i]][src[j]]
  const long long ldm = s2;
  TE *M = tk.M;
  if (form == 1) {
    for (int e = tid; e < s * s; e += kNodeThreads) {
      const int i = e % s, j = e / s;
      M[i + (long long)j * ldm] = TE(A[at[i] * lda + src[j]]);
    }
    return;
  }
  // form 0: the blocks of M around S^{-1} (r0 x r0)
  for (int e = tid; e < r0 * r0; e += kNodeThreads) {
    const int i = e % r0, j = e / r0;
    M[i + (long long)(r1 + j) * ldm] = TE(A[at[i] * lda + src[j]]);
  }
  if (stage) {
    for (int e = tid; e < r0 * r0; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      Ss[e] = A[at[i] * lda + src[j]];
    }
    __syncthreads();
    // G0 = -S^{-1} V1Tu1 (r0 x r1): M's upper left block, kept for the last product
    node_product_dmma(r0, r1, r0, -1.0, false, Ss, r0, W1s, r0, [&](int i, int c, double v) {
      Gs[i + c * r0] = v;
      M[i + (long long)c * ldm] = TE(v);
    });
    // -V0Tu0 S^{-1} (r1 x r0): M's lower right block
    node_product_dmma(r1, r0, r0, -1.0, false, W0s, r1, Ss, r0, [&](int i, int c, double v) {
      M[(r0 + i) + (long long)(r1 + c) * ldm] = TE(v);
    });
    __syncthreads();
    // I - V0Tu0 G0 (r1 x r1): M's lower left block
    node_product_dmma(r1, r1, r0, -1.0, true, W0s, r1, Gs, r0, [&](int i, int c, double v) {
      M[(r0 + i) + (long long)c * ldm] = TE(v);
    });
    return;
  }
  const TW *W0u = tk.W0u, *W1u = tk.W1u;
  const long long l0 = tk.ldw0u, l1 = tk.ldw1u;
  double *F = tk.F;
  // F = -V0Tu0 S^{-1} (r1 x r0): M's lower right block and FP64 work copy
  node_product(
      r1, r0, r0, -1.0, false, [&](int i, int k) { return double(W0u[i + k * l0]); },
      [&](int k, int c) { return A[at[k] * lda + src[c]]; },
      [&](int i, int c, double v) {
        F[i + (long long)c * r1] = v;
        M[(r0 + i) + (long long)(r1 + c) * ldm] = TE(v);
      });
  // G0 = -S^{-1} V1Tu1 (r0 x r1): M's upper left block
  node_product(
      r0, r1, r0, -1.0, false, [&](int i, int k) { return A[at[i] * lda + src[k]]; },
      [&](int k, int c) { return double(W1u[k + c * l1]); },
      [&](int i, int c, double v) { M[i + (long long)c * ldm] = TE(v); });
  __syncthreads();  // F (global) visible to the whole CTA
  // I - V0Tu0 G0 = I + V0Tu0 S^{-1} V1Tu1 = I - F V1Tu1 (r1 x r1): M's lower left block
  node_product(
      r1, r1, r0, -1.0, true, [&](int i, int k) { return F[i + (long long)k * r1]; },
      [&](int k, int c) { return double(W1u[k + c * l1]); },
      [&](int i, int c, double v) { M[(r0 + i) + (long long)c * ldm] = TE(v); });
}

}  // namespace

size_t node_factor_smem(int max_s) { return node_factor_words(max_s) * sizeof(double); }

bool node_factor_stages(int max_s, int max_r) {
  return node_factor_smem(max_s) + 4 * (size_t)max_r * max_r * sizeof(double) <= 200 * 1024;
}

template <typename TW, typename TE>
void launch_node_factor(const NodeTask<TW, TE> *tasks, int count, int max_s, int max_r, int form,
                        int *info, cudaStream_t s, bool g_alias) {
  if (count <= 0) return;
  size_t smem = node_factor_smem(max_s);
  const int stage = (form == 0 && node_factor_stages(max_s, max_r)) ? 1 : 0;
  const int galias = (stage && g_alias) ? 1 : 0;
  // staged: V0Tu0, V1Tu1 (TW), then S^{-1} and, unless it reuses A, G0
  // (FP64); the register elimination's scratch (s <= 64) shares the latter
  const size_t tail = std::max(
      stage ? (size_t)max_r * max_r * (galias ? 1 : 2) * sizeof(double) : (size_t)0,
      max_s <= 64 ? kGjScratchWords * sizeof(double) : (size_t)0);
  if (stage) smem += (size_t)max_r * max_r * 2 * sizeof(TW);
  smem += tail;
  auto go = [&](auto kern) {
    raise_smem_limit(reinterpret_cast<const void *>(kern), smem);
    // the largest shared-memory carveout: two CTAs of up to ~110 KB per SM
    HODLR_CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void *>(kern),
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared));
    kern<<<count, kNodeThreads, smem, s>>>(tasks, form, max_s, max_r, stage, galias, info);
  };
  if (max_s <= 32) go(node_factor_kernel<TW, TE, 1>);
  else if (max_s <= 64) go(node_factor_kernel<TW, TE, 2>);
  else go(node_factor_kernel<TW, TE, (kMaxNodeS + 31) / 32>);
  HODLR_LAUNCH_CHECK();
}

template void launch_node_factor<double, double>(const NodeTask<double, double> *, int, int,
                                                 int, int, int *, cudaStream_t, bool);
template void launch_node_factor<float, float>(const NodeTask<float, float> *, int, int, int,
                                               int, int *, cudaStream_t, bool);

}  // namespace hodlr
