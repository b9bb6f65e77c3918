// gemm_dmma.cu -- batched FP64 GEMM items (N > 32) on the FP64 tensor-core
// instruction mma.sync.m16n8k4.f64 (DMMA).
//
// The plain FP64 path (the reference's arithmetic: dgemm in the leaf solve's
// blocked LU, the reduce V^T [d | u] of gemm.cc:315-384 and the broadcast
// d -= u eta of gemm.cc:417-478) runs every wide product through this kernel:
//   C = beta Cin + alpha sum_s op(A_s) B_s,  op(A) = A (M x K) or A^T (A K x M).
// One CTA computes a BM x 128 tile of one item (BM = 64, two CTAs per SM, or
// 128 for items of at most 128 rows), 8 warps in a 2 x 4 grid, each warp a
// (BM / 2) x 32 block as (BM / 32) x 4 DMMA tiles of 16 x 8; K advances 16 at a time through a 3-stage cp.async ring (16-byte
// copies where the addresses allow, zero fill outside the item).  One DMMA
// does the work of 512 FP64 FMAs, so the kernel is bound by the FP64 pipe
// rather than by instruction issue.  Shared-memory layouts (doubles):
//   op(A) = A:    As[k][m], row stride BM + 4   (m contiguous, like A)
//   op(A) = A^T:  As[m][k], row stride 20       (k contiguous, like A)
//   B:            Bs[n][k], row stride 20       (k contiguous, like B)
// The strides put the 16 lanes of each half-warp's fragment loads in 16
// distinct 8-byte bank slots.  For the in-place updates (alpha = +-1,
// beta = 1) the accumulators start from alpha * Cin, so the C tile's loads
// overlap the main loop: alpha * (alpha * c + s) == c + alpha * s exactly.
#include "common.cuh"
#include "gemm_dmma.cuh"

namespace hodlr {

namespace {

constexpr int kThreads = 256;
constexpr int BN = 128, BK = 16, kStages = 3;
constexpr int LDK = BK + 4;  // k-contiguous row stride (doubles)

__device__ inline void cpa(void *dst, const void *src, int bytes, bool ok) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = ok ? bytes : 0;
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n));
}
__device__ inline void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Fragments of m16n8k4 .f64 (g = lane / 4, t = lane % 4): A a0 = A[g][t],
// a1 = A[g + 8][t]; B b = B[t][g]; C c0..c3 = C[g][2t], C[g][2t + 1],
// C[g + 8][2t], C[g + 8][2t + 1].
__device__ inline void dmma(double (&c)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
      "{%0, %1, %2, %3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b));
}

template <int BM, bool TRANS>
constexpr int a_stage_doubles() {
  return TRANS ? BM * LDK : BK * (BM + 4);
}
constexpr int b_stage_doubles() { return BN * LDK; }

template <int BM, bool TRANS>
__global__ void __launch_bounds__(kThreads, BM == 64 ? 2 : 1)
    gemm_dmma_tile_kernel(const GemmItem<double, double> *__restrict__ items,
                          const GemmSeg<double> *__restrict__ segs, double alpha, double beta,
                          int mtiles, int ntiles) {
  constexpr int MT = BM / 32;          // 16-row DMMA tiles per warp
  constexpr int AP = BM + 4;           // As[k][m] row stride (non-trans)
  constexpr int AS = a_stage_doubles<BM, TRANS>(), BS = b_stage_doubles();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);
  double *Bs = As + (size_t)kStages * AS;
  // one-dimensional grid, the tiles of an item consecutive (column tiles
  // fastest): CTAs resident together share the item's A rows and B columns
  // through L2
  const int per = mtiles * ntiles;
  const int itx = blockIdx.x / per, rem = blockIdx.x - itx * per;
  const GemmItem<double, double> it = items[itx];
  const int m0 = (rem / ntiles) * BM, n0 = (rem % ntiles) * BN;
  if (m0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * (BM / 2), wn = (warp & 3) * 32;

  double acc[MT][4][4];
  const bool preload = it.Cin && beta == 1.0 && (alpha == 1.0 || alpha == -1.0);
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        double x = 0.0;
        if (preload) {
          const int row = m0 + wm + mt * 16 + g + (v >> 1) * 8;
          const int col = n0 + wn + nt * 8 + 2 * t + (v & 1);
          if (row < it.M && col < it.N) x = alpha * it.Cin[row + (long long)col * it.ldcin];
        }
        acc[mt][nt][v] = x;
      }

  // the item's K stages, flattened over its segments
  int s_cur = it.seg_begin;
  const int s_end = it.seg_begin + it.seg_count;
  GemmSeg<double> sg{};
  int k0 = 0;
  bool valid = false;
  auto settle = [&](int &s, GemmSeg<double> &g_, int &k, bool &ok) {
    ok = false;
    for (; s < s_end; ++s) {
      g_ = segs[s];
      if (g_.K > 0) { ok = true; k = 0; return; }
    }
  };
  settle(s_cur, sg, k0, valid);
  int ls = s_cur, lk = k0;
  GemmSeg<double> lsg = sg;
  bool lvalid = valid;
  auto advance = [&](int &s, GemmSeg<double> &g_, int &k, bool &ok) {
    k += BK;
    if (k < g_.K) return;
    ++s;
    settle(s, g_, k, ok);
  };

  auto load = [&](int stage) {
    if (lvalid) {
      double *a = As + (size_t)stage * AS;
      double *b = Bs + (size_t)stage * BS;
      const double *A = lsg.A, *B = lsg.B;
      const long long lda = lsg.lda, ldb = lsg.ldb;
      const int K = lsg.K;
      if (!TRANS) {
        // As[k][m]: BK rows of BM doubles, m contiguous in A
        const bool vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((lda & 1) == 0) &&
                         ((m0 & 1) == 0);
#pragma unroll
        for (int e = tid; e < BK * (BM / 2); e += kThreads) {
          const int k = e / (BM / 2), mv = 2 * (e % (BM / 2));
          const int gk = lk + k, gm = m0 + mv;
          const double *src = A + gm + (long long)gk * lda;
          double *dst = a + k * AP + mv;
          if (vec && gk < K && gm + 2 <= it.M) {
            cpa(dst, src, 16, true);
          } else {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const bool ok = gk < K && gm + u < it.M;
              cpa(dst + u, ok ? src + u : A, 8, ok);
            }
          }
        }
      } else {
        // As[m][k]: BM rows of BK doubles, k contiguous in A
        const bool vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((lda & 1) == 0) &&
                         ((lk & 1) == 0);
#pragma unroll
        for (int e = tid; e < BM * (BK / 2); e += kThreads) {
          const int m = e / (BK / 2), kv = 2 * (e % (BK / 2));
          const int gk = lk + kv, gm = m0 + m;
          const double *src = A + gk + (long long)gm * lda;
          double *dst = a + m * LDK + kv;
          if (vec && gm < it.M && gk + 2 <= K) {
            cpa(dst, src, 16, true);
          } else {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const bool ok = gm < it.M && gk + u < K;
              cpa(dst + u, ok ? src + u : A, 8, ok);
            }
          }
        }
      }
      // Bs[n][k]: BN rows of BK doubles, k contiguous in B
      const bool vecb = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && ((ldb & 1) == 0) &&
                        ((lk & 1) == 0);
#pragma unroll
      for (int e = tid; e < BN * (BK / 2); e += kThreads) {
        const int n = e / (BK / 2), kv = 2 * (e % (BK / 2));
        const int gk = lk + kv, gn = n0 + n;
        const double *src = B + gk + (long long)gn * ldb;
        double *dst = b + n * LDK + kv;
        if (vecb && gn < it.N && gk + 2 <= K) {
          cpa(dst, src, 16, true);
        } else {
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const bool ok = gn < it.N && gk + u < K;
            cpa(dst + u, ok ? src + u : B, 8, ok);
          }
        }
      }
      advance(ls, lsg, lk, lvalid);
    }
    cpa_commit();
  };

#pragma unroll
  for (int i = 0; i < kStages - 1; ++i) load(i);
  int st = 0, lst = kStages - 1;
  while (valid) {
    load(lst);
    lst = lst + 1 == kStages ? 0 : lst + 1;
    cpa_wait<kStages - 1>();
    __syncthreads();
    const double *a = As + (size_t)st * AS;
    const double *b = Bs + (size_t)st * BS;
#pragma unroll
    for (int ks = 0; ks < BK; ks += 4) {
      double bv[4];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) bv[nt] = b[(wn + nt * 8 + g) * LDK + ks + t];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int mr = wm + mt * 16 + g;
        const double a0 = TRANS ? a[mr * LDK + ks + t] : a[(ks + t) * AP + mr];
        const double a1 = TRANS ? a[(mr + 8) * LDK + ks + t] : a[(ks + t) * AP + mr + 8];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], a0, a1, bv[nt]);
      }
    }
    __syncthreads();  // stage st is refilled kStages - 1 tiles later
    st = st + 1 == kStages ? 0 : st + 1;
    advance(s_cur, sg, k0, valid);
  }
  cpa_wait<0>();

#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = m0 + wm + mt * 16 + g + (v >> 1) * 8;
        const int col = n0 + wn + nt * 8 + 2 * t + (v & 1);
        if (row < it.M && col < it.N) {
          double x = alpha * acc[mt][nt][v];
          if (it.Cin && !preload) x += beta * it.Cin[row + (long long)col * it.ldcin];
          it.C[row + (long long)col * it.ldc] = x;
        }
      }
}

template <int BM, bool TRANS>
void launch_bm(const GemmItem<double, double> *items, const GemmSeg<double> *segs, int nitems,
               int max_m, int max_n, double alpha, double beta, cudaStream_t s) {
  const size_t smem =
      (size_t)kStages * (a_stage_doubles<BM, TRANS>() + b_stage_doubles()) * sizeof(double);
  raise_smem_limit(reinterpret_cast<const void *>(gemm_dmma_tile_kernel<BM, TRANS>), smem);
  const int mt = cdiv(max_m, BM), nt = cdiv(max_n, BN);
  const long long total = (long long)nitems * mt * nt;
  if (total > 0x7fffffffLL) throw CudaError{cudaErrorInvalidConfiguration};
  gemm_dmma_tile_kernel<BM, TRANS>
      <<<(unsigned)total, kThreads, smem, s>>>(items, segs, alpha, beta, mt, nt);
  HODLR_LAUNCH_CHECK();
}

}  // namespace

void launch_dmma_tile(const GemmItem<double, double> *items, const GemmSeg<double> *segs,
                      int nitems, int max_m, int max_n, bool trans, double alpha, double beta,
                      cudaStream_t s) {
  if (nitems <= 0 || max_m <= 0 || max_n <= 0) return;
  // Items of at most 128 rows run as one tile row of 128: the leaf LU's
  // block-row solves compute C = L^{-1} C in place (C is also the B operand),
  // which is only correct when a single CTA reads all of C's rows before it
  // writes any.  Taller items (the trailing updates, the broadcast) are never
  // in place and take 64-row tiles: two CTAs per SM, so one CTA's C loads and
  // stores overlap the other's DMMAs (a 128-row tile needs ~250 registers per
  // thread and runs alone on its SM).
  if (max_m > 64 && max_m <= 128) {
    if (trans) launch_bm<128, true>(items, segs, nitems, max_m, max_n, alpha, beta, s);
    else launch_bm<128, false>(items, segs, nitems, max_m, max_n, alpha, beta, s);
  } else {
    if (trans) launch_bm<64, true>(items, segs, nitems, max_m, max_n, alpha, beta, s);
    else launch_bm<64, false>(items, segs, nitems, max_m, max_n, alpha, beta, s);
  }
}

}  // namespace hodlr
