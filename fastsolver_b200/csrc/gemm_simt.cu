// gemm_simt.cu -- batched multi-segment GEMM on the FP64 / FP32 pipes.
//
// One launch computes every item of a tree level:
//   C = beta * Cin + alpha * sum_s op(A_s) B_s
// which covers the three GEMM call sites of fastSolver's solve:
//   * GEMM_Reduce_Task  (src/solver/gemm.cc:364-380: W += V^T U[:, cols]),
//     as split-K items over row chunks, each writing one partial-sum slot that
//     the node kernel later sums in a fixed order (the REDOP_ADD reduction of
//     gemm.cc:74-133 without floating-point atomics);
//   * GEMM_Broadcast_Task (gemm.cc:464-477: d = d - u eta), in place;
//   * the HODLR matvec's r = b - D x - sum_d U_d t_d (one segment per term).
//
// Tile 64 x 128 x 16 (64 x 32 x 16 for items of at most 32 columns) per
// CTA, 256 threads, 4 x 8 (4 x 2) register tile per thread,
// operands staged through shared memory with a one-tile register prefetch.
#include "common.cuh"
#include "gemm_simt.cuh"

namespace hodlr {

namespace {

constexpr int BM = 64, BK = 16, NT = 256;
constexpr int APAD = BM + 4;

// BN = 16 * TN columns per CTA (TN = 8: wide items, TN = 2: m-column sweeps)
template <typename TA, typename TC, typename TACC, bool TRANS, int TN>
__global__ void __launch_bounds__(NT)
    gemm_items_kernel(const GemmItem<TA, TC> *__restrict__ items,
                      const GemmSeg<TA> *__restrict__ segs, TACC alpha, TACC beta) {
  constexpr int BN = 16 * TN, BPAD = BN + 4, NB = BK * BN / NT;
  __shared__ __align__(16) TACC As[BK * APAD];
  __shared__ __align__(16) TACC Bs[BK * BPAD];
  const GemmItem<TA, TC> it = items[blockIdx.x];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.z * BN;
  if (m0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x;
  const int tr = tid & 15, tc = tid >> 4;

  TACC acc[4][TN];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = TACC(0);

  TACC ra[4], rb[NB];
  for (int s = it.seg_begin; s < it.seg_begin + it.seg_count; ++s) {
    const GemmSeg<TA> sg = segs[s];
    const int K = sg.K;
    auto load = [&](int k0) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int idx = tid + NT * i;
        int k, m;
        if (TRANS) { k = idx & (BK - 1); m = idx >> 4; }
        else { m = idx & (BM - 1); k = idx >> 6; }
        const int gk = k0 + k, gm = m0 + m;
        ra[i] = (gk < K && gm < it.M)
                    ? TACC(TRANS ? sg.A[gk + (long long)gm * sg.lda] : sg.A[gm + (long long)gk * sg.lda])
                    : TACC(0);
      }
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const int idx = tid + NT * i;
        const int k = idx & (BK - 1), n = idx >> 4;
        const int gk = k0 + k, gn = n0 + n;
        rb[i] = (gk < K && gn < it.N) ? TACC(sg.B[gk + (long long)gn * sg.ldb]) : TACC(0);
      }
    };
    if (K <= 0) continue;
    load(0);
    for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int idx = tid + NT * i;
        int k, m;
        if (TRANS) { k = idx & (BK - 1); m = idx >> 4; }
        else { m = idx & (BM - 1); k = idx >> 6; }
        As[k * APAD + m] = ra[i];
      }
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const int idx = tid + NT * i;
        Bs[(idx & (BK - 1)) * BPAD + (idx >> 4)] = rb[i];
      }
      __syncthreads();
      if (k0 + BK < K) load(k0 + BK);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        TACC a[4], b[TN];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[kk * APAD + tr * 4 + i];
#pragma unroll
        for (int j = 0; j < TN; ++j) b[j] = Bs[kk * BPAD + tc * TN + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] += a[i] * b[j];
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < TN; ++j) {
    const int gn = n0 + tc * TN + j;
    if (gn >= it.N) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int gm = m0 + tr * 4 + i;
      if (gm >= it.M) continue;
      TACC v = alpha * acc[i][j];
      if (it.Cin) v += beta * TACC(it.Cin[gm + (long long)gn * it.ldcin]);
      it.C[gm + (long long)gn * it.ldc] = TC(v);
    }
  }
}


// ---------------------------------------------------------------------------
// Skinny items (N <= 32 columns: the m right-hand sides of the matvec and of
// the refinement sweeps).  These are bandwidth-bound, so the kernels aim at
// bytes in flight rather than register tiles.
// ---------------------------------------------------------------------------

// NN: one thread per output row, N accumulators; B's rows staged in shared
// memory (broadcast reads), A streamed with 8 loads in flight per thread.
template <typename TA, typename TC, typename TACC, int NC>
__global__ void __launch_bounds__(NT)
    skinny_nn_kernel(const GemmItem<TA, TC> *__restrict__ items,
                     const GemmSeg<TA> *__restrict__ segs, TACC alpha, TACC beta) {
  constexpr int KT = 64;
  __shared__ __align__(16) TACC Bs[KT * NC];
  const GemmItem<TA, TC> it = items[blockIdx.x];
  const int m0 = blockIdx.y * NT;
  if (m0 >= it.M) return;
  const int tid = threadIdx.x;
  const int row = m0 + tid;
  TACC acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = TACC(0);
  for (int s = it.seg_begin; s < it.seg_begin + it.seg_count; ++s) {
    const GemmSeg<TA> sg = segs[s];
    for (int k0 = 0; k0 < sg.K; k0 += KT) {
      const int kt = min(KT, sg.K - k0);
      for (int e = tid; e < KT * NC; e += NT) {
        const int kk = e % KT, c = e / KT;
        Bs[kk * NC + c] = (kk < kt && c < it.N) ? TACC(sg.B[(k0 + kk) + (long long)c * sg.ldb])
                                                : TACC(0);
      }
      __syncthreads();
      if (row < it.M) {
        const TA *a = sg.A + row + (long long)k0 * sg.lda;
        int kk = 0;
        for (; kk + 8 <= kt; kk += 8) {
          TACC av[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) av[u] = TACC(a[(long long)(kk + u) * sg.lda]);
#pragma unroll
          for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int c = 0; c < NC; ++c) acc[c] += av[u] * Bs[(kk + u) * NC + c];
        }
        for (; kk < kt; ++kk) {
          const TACC av = TACC(a[(long long)kk * sg.lda]);
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[c] += av * Bs[kk * NC + c];
        }
      }
      __syncthreads();
    }
  }
  if (row < it.M) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (c >= it.N) break;
      TACC v = alpha * acc[c];
      if (it.Cin) v += beta * TACC(it.Cin[row + (long long)c * it.ldcin]);
      it.C[row + (long long)c * it.ldc] = TC(v);
    }
  }
}

// TN: C (64 x 16 tile) = A^T B over the item's K rows.  Tiles of 64 rows are
// staged in shared memory; warp w takes rows w, w+8, ... of each tile with a
// 4 x 8 register tile per lane; the 8 warp partials are summed at the end.
template <typename TA, typename TC, typename TACC>
__global__ void __launch_bounds__(NT)
    skinny_tn_kernel(const GemmItem<TA, TC> *__restrict__ items,
                     const GemmSeg<TA> *__restrict__ segs, TACC alpha, TACC beta) {
  constexpr int TM = 64, TNc = 16, KT = 64;
  __shared__ __align__(16) TACC As[KT * TM];
  __shared__ __align__(16) TACC Bs[KT * TNc];
  extern __shared__ __align__(16) unsigned char red_raw[];
  TACC *red = reinterpret_cast<TACC *>(red_raw);  // 8 x (TM * TNc)
  const GemmItem<TA, TC> it = items[blockIdx.x];
  const int m0 = blockIdx.y * TM, n0 = blockIdx.z * TNc;
  if (m0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int mg = lane & 15, ng = lane >> 4;  // m = mg*4.., n = ng*8..
  TACC acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = TACC(0);
  for (int s = it.seg_begin; s < it.seg_begin + it.seg_count; ++s) {
    const GemmSeg<TA> sg = segs[s];
    for (int k0 = 0; k0 < sg.K; k0 += KT) {
      // A tile: rows k0.., columns m0..m0+63; threads run along k (coalesced)
#pragma unroll
      for (int u = 0; u < KT * TM / NT; ++u) {
        const int e = tid + u * NT;
        const int kk = e % KT, mm = e / KT;
        const int gk = k0 + kk, gm = m0 + mm;
        As[kk * TM + mm] =
            (gk < sg.K && gm < it.M) ? TACC(sg.A[gk + (long long)gm * sg.lda]) : TACC(0);
      }
#pragma unroll
      for (int u = 0; u < KT * TNc / NT; ++u) {
        const int e = tid + u * NT;
        const int kk = e % KT, nn = e / KT;
        const int gk = k0 + kk, gn = n0 + nn;
        Bs[kk * TNc + nn] =
            (gk < sg.K && gn < it.N) ? TACC(sg.B[gk + (long long)gn * sg.ldb]) : TACC(0);
      }
      __syncthreads();
#pragma unroll 2
      for (int kk = warp; kk < KT; kk += 8) {
        TACC a[4], b[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[kk * TM + mg * 4 + i];
#pragma unroll
        for (int j = 0; j < 8; ++j) b[j] = Bs[kk * TNc + ng * 8 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j)
      red[warp * (TM * TNc) + (ng * 8 + j) * TM + mg * 4 + i] = acc[i][j];
  __syncthreads();
  for (int e = tid; e < TM * TNc; e += NT) {
    const int mm = e % TM, nn = e / TM;
    const int gm = m0 + mm, gn = n0 + nn;
    if (gm >= it.M || gn >= it.N) continue;
    TACC v = TACC(0);
#pragma unroll
    for (int w = 0; w < 8; ++w) v += red[w * (TM * TNc) + e];
    v *= alpha;
    if (it.Cin) v += beta * TACC(it.Cin[gm + (long long)gn * it.ldcin]);
    it.C[gm + (long long)gn * it.ldc] = TC(v);
  }
}

}  // namespace

template <typename TA, typename TC, typename TACC>
void launch_gemm_items(const GemmItem<TA, TC> *items, const GemmSeg<TA> *segs, int nitems,
                       int max_m, int max_n, bool trans, TACC alpha, TACC beta,
                       cudaStream_t s) {
  if (nitems <= 0 || max_m <= 0 || max_n <= 0) return;
  if (max_n <= 32) {
    if (trans) {
      dim3 grid(nitems, cdiv(max_m, 64), cdiv(max_n, 16));
      const size_t red = 8 * 64 * 16 * sizeof(TACC);
      HODLR_CUDA_TRY(cudaFuncSetAttribute(skinny_tn_kernel<TA, TC, TACC>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)red));
      skinny_tn_kernel<TA, TC, TACC><<<grid, NT, red, s>>>(items, segs, alpha, beta);
    } else {
      dim3 grid(nitems, cdiv(max_m, NT));
      if (max_n <= 16)
        skinny_nn_kernel<TA, TC, TACC, 16><<<grid, NT, 0, s>>>(items, segs, alpha, beta);
      else
        skinny_nn_kernel<TA, TC, TACC, 32><<<grid, NT, 0, s>>>(items, segs, alpha, beta);
    }
  } else {
    dim3 grid(nitems, cdiv(max_m, BM), cdiv(max_n, 128));
    if (trans)
      gemm_items_kernel<TA, TC, TACC, true, 8><<<grid, NT, 0, s>>>(items, segs, alpha, beta);
    else
      gemm_items_kernel<TA, TC, TACC, false, 8><<<grid, NT, 0, s>>>(items, segs, alpha, beta);
  }
  HODLR_LAUNCH_CHECK();
}

template void launch_gemm_items<double, double, double>(const GemmItem<double, double> *,
                                                        const GemmSeg<double> *, int, int,
                                                        int, bool, double, double,
                                                        cudaStream_t);
template void launch_gemm_items<float, double, double>(const GemmItem<float, double> *,
                                                       const GemmSeg<float> *, int, int, int,
                                                       bool, double, double, cudaStream_t);
template void launch_gemm_items<float, float, float>(const GemmItem<float, float> *,
                                                     const GemmSeg<float> *, int, int, int,
                                                     bool, float, float, cudaStream_t);

}  // namespace hodlr
