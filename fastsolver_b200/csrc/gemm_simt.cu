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
#include <type_traits>

#include <cstdlib>

#include "common.cuh"
#include "gemm_dmma.cuh"
#include "gemm_simt.cuh"
#include "gemm_skinny.cuh"
#include "tc_gemm.cuh"

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
    // the column's Cin values before its stores (C may alias Cin)
    TC cin[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int gm = m0 + tr * 4 + i;
      cin[i] = (it.Cin && gm < it.M) ? it.Cin[gm + (long long)gn * it.ldcin] : TC(0);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int gm = m0 + tr * 4 + i;
      if (gm >= it.M) continue;
      TACC v = alpha * acc[i][j];
      if (it.Cin) v += beta * TACC(cin[i]);
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
    // the row's Cin values before its stores (C may alias Cin)
    TC cin[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c)
      cin[c] = (it.Cin && c < it.N) ? it.Cin[row + (long long)c * it.ldcin] : TC(0);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (c >= it.N) break;
      TACC v = alpha * acc[c];
      if (it.Cin) v += beta * TACC(cin[c]);
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

// ---------------------------------------------------------------------------
// Tiled items (N > 32): BM x 128 tile per CTA (BM = 64 or 128), 256 threads,
// TM x 8 register tile per thread (thread x -> rows, y -> columns, so the
// epilogue's column-major accesses coalesce), K staged in BK-deep slices through a
// two-stage cp.async pipeline.  Register fragments are interleaved in
// 16-byte vectors (2 doubles / 4 floats) so that the shared-memory reads of
// the 16 row groups of a warp are contiguous (no bank conflicts) and the
// column fragments are warp-broadcasts.
// ---------------------------------------------------------------------------

__device__ inline void cp_async_elem(void *smem, const void *gmem, int bytes, bool pred) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int n = pred ? bytes : 0;
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ inline void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

template <typename T, typename TC, bool TRANS, int BM>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 2 : 1)
    gemm_tile_kernel(const GemmItem<T, TC> *__restrict__ items,
                     const GemmSeg<T> *__restrict__ segs, T alpha, T beta) {
  constexpr int BN = 128;
  constexpr int BK = sizeof(T) == 8 ? 8 : 16;
  constexpr int VW = 16 / sizeof(T);       // elements per 16-byte vector
  constexpr int TM = BM / 16, TN = BN / 16;
  constexpr int AP = BM + 4, BP = BN + 4;  // padded row strides (16-byte multiples)
  constexpr int NA = BK * BM / NT, NBL = BK * BN / NT;
  __shared__ __align__(16) T As[2][BK * AP];
  __shared__ __align__(16) T Bs[2][BK * BP];
  const GemmItem<T, TC> it = items[blockIdx.x];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.z * BN;
  if (m0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;

  T acc[TM][TN];
  // alpha = +-1, beta = 1 (the in-place updates): start from alpha * Cin so the
  // C loads overlap the main loop; alpha * (alpha * c + s) == c + alpha * s exactly
  const bool preload = it.Cin && beta == T(1) && (alpha == T(1) || alpha == T(-1));
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      T v = T(0);
      if (preload) {
        const int gm = m0 + (i / VW) * (16 * VW) + tx * VW + (i % VW);
        const int gn = n0 + (j / VW) * (16 * VW) + ty * VW + (j % VW);
        if (gm < it.M && gn < it.N) v = alpha * T(it.Cin[gm + (long long)gn * it.ldcin]);
      }
      acc[i][j] = v;
    }

  for (int sgi = it.seg_begin; sgi < it.seg_begin + it.seg_count; ++sgi) {
    const GemmSeg<T> sg = segs[sgi];
    const int K = sg.K;
    if (K <= 0) continue;
    const int ntiles = (K + BK - 1) / BK;
    auto issue = [&](int kt, int buf) {
      const int k0 = kt * BK;
#pragma unroll
      for (int u = 0; u < NA; ++u) {
        const int idx = tid + u * NT;
        int k, m;
        if (TRANS) { k = idx % BK; m = idx / BK; }
        else { m = idx % BM; k = idx / BM; }
        const int gk = k0 + k, gm = m0 + m;
        const bool ok = gk < K && gm < it.M;
        const T *src = ok ? (TRANS ? sg.A + gk + (long long)gm * sg.lda
                                   : sg.A + gm + (long long)gk * sg.lda)
                          : sg.A;
        cp_async_elem(&As[buf][k * AP + m], src, sizeof(T), ok);
      }
#pragma unroll
      for (int u = 0; u < NBL; ++u) {
        const int idx = tid + u * NT;
        const int k = idx % BK, n = idx / BK;
        const int gk = k0 + k, gn = n0 + n;
        const bool ok = gk < K && gn < it.N;
        const T *src = ok ? sg.B + gk + (long long)gn * sg.ldb : sg.B;
        cp_async_elem(&Bs[buf][k * BP + n], src, sizeof(T), ok);
      }
    };
    issue(0, 0);
    cp_async_commit();
    for (int kt = 0; kt < ntiles; ++kt) {
      if (kt + 1 < ntiles) issue(kt + 1, (kt + 1) & 1);
      cp_async_commit();
      cp_async_wait1();
      __syncthreads();
      const T *Ab = As[kt & 1];
      const T *Bb = Bs[kt & 1];
      using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        T a[TM], b[TN];
#pragma unroll
        for (int g = 0; g < TM / VW; ++g) {
          const V va = *reinterpret_cast<const V *>(Ab + kk * AP + g * (16 * VW) + tx * VW);
          const T *pv = reinterpret_cast<const T *>(&va);
#pragma unroll
          for (int v = 0; v < VW; ++v) a[g * VW + v] = pv[v];
        }
#pragma unroll
        for (int g = 0; g < TN / VW; ++g) {
          const V vb = *reinterpret_cast<const V *>(Bb + kk * BP + g * (16 * VW) + ty * VW);
          const T *pv = reinterpret_cast<const T *>(&vb);
#pragma unroll
          for (int v = 0; v < VW; ++v) b[g * VW + v] = pv[v];
        }
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] += a[i] * b[j];
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < TN; ++j) {
    const int gn = n0 + (j / VW) * (16 * VW) + ty * VW + (j % VW);
    if (gn >= it.N) continue;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int gm = m0 + (i / VW) * (16 * VW) + tx * VW + (i % VW);
      if (gm >= it.M) continue;
      T v = alpha * acc[i][j];
      if (it.Cin && !preload) v += beta * T(it.Cin[gm + (long long)gn * it.ldcin]);
      it.C[gm + (long long)gn * it.ldc] = TC(v);
    }
  }
}

}  // namespace

// FP32 GEMM items (N > 32) run on the tensor cores unless HODLR_TC=0.
bool tc_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("HODLR_TC");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename TA, typename TC, typename TACC>
void launch_gemm_items(const GemmItem<TA, TC> *items, const GemmSeg<TA> *segs, int nitems,
                       int max_m, int max_n, bool trans, TACC alpha, TACC beta,
                       cudaStream_t s, bool allow_tc) {
  if (nitems <= 0 || max_m <= 0 || max_n <= 0) return;
  if (max_n <= 32 && std::is_same<TA, TC>::value && std::is_same<TA, TACC>::value) {
    using T = TACC;
    launch_skinny<T>(reinterpret_cast<const GemmItem<T, T> *>(items),
                     reinterpret_cast<const GemmSeg<T> *>(segs), nitems, max_m, max_n, trans,
                     alpha, beta, s);
    return;
  }
  if (max_n <= 32) {
    if (trans) {
      dim3 grid(nitems, cdiv(max_m, 64), cdiv(max_n, 16));
      const size_t red = 8 * 64 * 16 * sizeof(TACC);
      raise_smem_limit(reinterpret_cast<const void *>(skinny_tn_kernel<TA, TC, TACC>), red);
      skinny_tn_kernel<TA, TC, TACC><<<grid, NT, red, s>>>(items, segs, alpha, beta);
    } else {
      dim3 grid(nitems, cdiv(max_m, NT));
      if (max_n <= 16)
        skinny_nn_kernel<TA, TC, TACC, 16><<<grid, NT, 0, s>>>(items, segs, alpha, beta);
      else
        skinny_nn_kernel<TA, TC, TACC, 32><<<grid, NT, 0, s>>>(items, segs, alpha, beta);
    }
  } else if (std::is_same<TA, float>::value && std::is_same<TC, float>::value && allow_tc &&
             tc_enabled()) {
    launch_tc_gemm<float>(reinterpret_cast<const GemmItem<float, float> *>(items),
                          reinterpret_cast<const GemmSeg<float> *>(segs), nitems, max_m, max_n,
                          trans, float(alpha), float(beta), s);
    return;
  } else if (std::is_same<TA, double>::value && std::is_same<TC, double>::value &&
             std::is_same<TACC, double>::value) {
    launch_dmma_tile(reinterpret_cast<const GemmItem<double, double> *>(items),
                     reinterpret_cast<const GemmSeg<double> *>(segs), nitems, max_m, max_n,
                     trans, double(alpha), double(beta), s);
    return;
  } else if (std::is_same<TA, TACC>::value) {
    using T = TACC;
    const auto *it2 = reinterpret_cast<const GemmItem<T, TC> *>(items);
    const auto *sg2 = reinterpret_cast<const GemmSeg<T> *>(segs);
    if (max_m <= 64) {
      dim3 grid(nitems, cdiv(max_m, 64), cdiv(max_n, 128));
      if (trans) gemm_tile_kernel<T, TC, true, 64><<<grid, NT, 0, s>>>(it2, sg2, alpha, beta);
      else gemm_tile_kernel<T, TC, false, 64><<<grid, NT, 0, s>>>(it2, sg2, alpha, beta);
    } else {
      dim3 grid(nitems, cdiv(max_m, 128), cdiv(max_n, 128));
      if (trans) gemm_tile_kernel<T, TC, true, 128><<<grid, NT, 0, s>>>(it2, sg2, alpha, beta);
      else gemm_tile_kernel<T, TC, false, 128><<<grid, NT, 0, s>>>(it2, sg2, alpha, beta);
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
                                                        cudaStream_t, bool);
template void launch_gemm_items<float, double, double>(const GemmItem<float, double> *,
                                                       const GemmSeg<float> *, int, int, int,
                                                       bool, double, double, cudaStream_t, bool);
template void launch_gemm_items<float, float, float>(const GemmItem<float, float> *,
                                                     const GemmSeg<float> *, int, int, int,
                                                     bool, float, float, cudaStream_t, bool);

}  // namespace hodlr
