// tc_gemm.cu -- split-BF16 tensor-core GEMM engine (tcgen05, sm_100a).
//
// The mixed-precision path runs its GEMMs (leaf TRSM/trailing updates, the
// reduce V^T [d | u] and the broadcast d -= u eta) on the 5th-generation
// tensor cores.  FP32 operands are split as x = hi + lo with hi = bf16(x),
// lo = bf16(x - hi), and each product is accumulated in FP32 in tensor memory
// as  A_hi B_hi + A_hi B_lo + A_lo B_hi  (the lo*lo term, ~2^-16 relative, is
// dropped; FP64 iterative refinement recovers full accuracy).
//
// One CTA (128 threads) computes a 128 x BN tile of one item:
//   * every thread owns one row of the A tile and one (or two) rows of the B
//     tile, loads its 32 K-values per stage from global memory (coalesced
//     across threads for the M-contiguous operands, 128-byte rows for the
//     K-contiguous ones), keeps the next stage's values in registers while the
//     current one is converted, and writes hi/lo bf16 into the UMMA canonical
//     K-major layout (8-row x 16-byte core matrices, no swizzle);
//   * a 3-stage shared-memory ring; thread 0 issues the MMAs
//     (tcgen05.mma.cta_group::1.kind::f16, M = 128, N = BN, K = 16) and
//     tcgen05.commit arrives on the stage's mbarrier when the tensor cores are
//     done with it; producers wait on that barrier before reusing the stage;
//   * the accumulator lives in TMEM (BN columns, allocated per CTA); the
//     epilogue reads it with tcgen05.ld (32 lanes per warp) and writes
//     alpha * acc + beta * Cin to global memory.
// The reduce's V^T X (M = r small, N wide) runs "swapped": the UMMA M side is
// the item's N and the result is written transposed.
// Every mbarrier wait is bounded; on timeout the kernel raises g_tc_error,
// waits (bounded) for its own MMAs, frees its TMEM and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace hodlr {

__device__ int g_tc_error = 0;

namespace {

constexpr int kThreads = 128;
constexpr int BM = 128;    // UMMA M
constexpr int BK = 32;     // K per stage (two MMA k-steps of 16)
constexpr int STAGES = 3;
constexpr long long kSpinLimit = 1LL << 26;

__device__ inline uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ inline void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait for the completion of phase `parity`; false on timeout.
__device__ inline bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < kSpinLimit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ inline void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ inline void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ inline void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ inline uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  // base offset 0, lbo mode 0, layout type 0 (SWIZZLE_NONE)
  return d;
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
         | ((uint32_t)(N >> 3) << 17)    // N
         | ((uint32_t)(M >> 4) << 24);   // M
}

__device__ inline void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                uint32_t accumulate) {
  const uint32_t z = 0;  // disable-output-lane mask: all lanes written
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ inline void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// Canonical K-major offset (bytes) of element (row, k) inside one operand
// stage holding `rows` rows x BK k: [kstep][row/8][k-chunk][row%8][8 elems].
__device__ inline uint32_t kmajor_off(int rows, int row, int kchunk_global) {
  const int ks = kchunk_global >> 1, kc = kchunk_global & 1;
  return (uint32_t)(ks * (rows / 8) * 256 + (row >> 3) * 256 + kc * 128 + (row & 7) * 16);
}

// Split 8 FP32 values into hi / lo bf16 and store one 16-byte chunk of each.
__device__ inline void split_store8(const float *v, unsigned char *hi, unsigned char *lo,
                                    uint32_t off) {
  __nv_bfloat162 h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * q]);
    const __nv_bfloat16 h1 = __float2bfloat16_rn(v[2 * q + 1]);
    const __nv_bfloat16 l0 = __float2bfloat16_rn(v[2 * q] - __bfloat162float(h0));
    const __nv_bfloat16 l1 = __float2bfloat16_rn(v[2 * q + 1] - __bfloat162float(h1));
    h[q] = __halves2bfloat162(h0, h1);
    l[q] = __halves2bfloat162(l0, l1);
  }
  *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(h);
  *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(l);
}

// Loads BK K-values of one row of an operand into registers (zero padded).
// kcontig: element (row, k) at base[k + row * ld] (K contiguous), else at
// base[row + k * ld] (row contiguous).
__device__ inline void load_row(float (&v)[BK], const float *base, long long ld, bool kcontig,
                                int row, int rows_valid, int k0, int K) {
  if (row >= rows_valid) {
#pragma unroll
    for (int k = 0; k < BK; ++k) v[k] = 0.f;
    return;
  }
  if (kcontig) {
    const float *p = base + (long long)row * ld + k0;
    const bool full = (k0 + BK <= K) && ((reinterpret_cast<uintptr_t>(p) & 15) == 0);
    if (full) {
#pragma unroll
      for (int q = 0; q < BK / 4; ++q) {
        const float4 x = __ldg(reinterpret_cast<const float4 *>(p) + q);
        v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < BK; ++k) v[k] = (k0 + k < K) ? __ldg(p + k) : 0.f;
    }
  } else {
    const float *p = base + row + (long long)k0 * ld;
#pragma unroll
    for (int k = 0; k < BK; ++k) v[k] = (k0 + k < K) ? __ldg(p + (long long)k * ld) : 0.f;
  }
}

template <int BN, typename TC>
__global__ void __launch_bounds__(kThreads)
    tc_gemm_kernel(const GemmItem<float, TC> *__restrict__ items,
                   const GemmSeg<float> *__restrict__ segs, float alpha, float beta, int trans,
                   int swap) {
  constexpr int A_BYTES = BM * BK * 2;  // one of hi / lo
  constexpr int B_BYTES = BN * BK * 2;
  constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  constexpr int BROWS = BN / kThreads > 0 ? BN / kThreads : 1;  // B rows per thread
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar_empty[STAGES];
  __shared__ __align__(8) uint64_t bar_done;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;

  const GemmItem<float, TC> it = items[blockIdx.x];
  // UMMA-M side (rows of D) and UMMA-N side (columns of D)
  const int Mu = swap ? it.N : it.M;
  const int Nu = swap ? it.M : it.N;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.z * BN;
  if (m0 >= Mu || n0 >= Nu) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bar_empty[s], 1);
    mbar_init(&bar_done, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  const uint32_t idesc = instr_desc(BM, BN);

  // total K tiles over all segments
  int ntiles = 0;
  for (int s = it.seg_begin; s < it.seg_begin + it.seg_count; ++s)
    ntiles += (segs[s].K + BK - 1) / BK;

  // operand access for the current tile: the UMMA A operand has rows along
  // Mu, the UMMA B operand rows along Nu
  int seg = it.seg_begin, seg_k0 = 0;
  GemmSeg<float> sg = segs[seg];
  while (seg < it.seg_begin + it.seg_count - 1 && sg.K <= 0) sg = segs[++seg];
  auto advance = [&]() {
    seg_k0 += BK;
    while (seg < it.seg_begin + it.seg_count - 1 && seg_k0 >= sg.K) {
      ++seg;
      seg_k0 = 0;
      sg = segs[seg];
    }
  };
  // item operand A (op(A): M x K) and B (K x N); element access helpers
  // UMMA-A rows = item rows (M) unless swapped (then item columns N).
  float va[BK], vb[BROWS][BK];
  auto fetch = [&]() {
    const int K = sg.K;
    if (!swap) {
      // UMMA A = op(A): row m; trans: A[k + m*lda] (K contiguous), else A[m + k*lda]
      load_row(va, sg.A, sg.lda, trans != 0, m0 + tid, it.M, seg_k0, K);
#pragma unroll
      for (int r = 0; r < BROWS; ++r) {
        const int n = n0 + tid + r * kThreads;
        load_row(vb[r], sg.B, sg.ldb, true, n, (tid + r * kThreads < BN) ? it.N : -1, seg_k0, K);
      }
    } else {
      // D^T = B^T op(A)^T: UMMA A row = item column n of B (K contiguous),
      // UMMA B row = item row m of op(A) (trans: K contiguous)
      load_row(va, sg.B, sg.ldb, true, m0 + tid, it.N, seg_k0, K);
#pragma unroll
      for (int r = 0; r < BROWS; ++r) {
        const int m = n0 + tid + r * kThreads;
        load_row(vb[r], sg.A, sg.lda, trans != 0, m, (tid + r * kThreads < BN) ? it.M : -1,
                 seg_k0, K);
      }
    }
  };

  bool ok = true;
  bool committed_done = false;
  if (ntiles > 0) fetch();
  for (int kt = 0; kt < ntiles; ++kt) {
    const int st = kt % STAGES;
    unsigned char *base = smem + st * STAGE_BYTES;
    unsigned char *ahi = base, *alo = base + A_BYTES;
    unsigned char *bhi = base + 2 * A_BYTES, *blo = bhi + B_BYTES;
    if (kt >= STAGES) {
      if (!mbar_wait(&bar_empty[st], ((kt / STAGES) - 1) & 1)) ok = false;
    }
    if (!ok) atomicExch(&abort_sh, 1);
    // convert + store this thread's rows
#pragma unroll
    for (int c = 0; c < BK / 8; ++c) split_store8(va + 8 * c, ahi, alo, kmajor_off(BM, tid, c));
#pragma unroll
    for (int r = 0; r < BROWS; ++r) {
      const int row = tid + r * kThreads;
      if (row < BN)
#pragma unroll
        for (int c = 0; c < BK / 8; ++c)
          split_store8(vb[r] + 8 * c, bhi, blo, kmajor_off(BN, row, c));
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    if (abort_sh) break;
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a_hi = smem_u32(ahi), a_lo = smem_u32(alo);
      const uint32_t b_hi = smem_u32(bhi), b_lo = smem_u32(blo);
#pragma unroll
      for (int ks = 0; ks < BK / 16; ++ks) {
        const uint32_t ao = ks * (BM / 8) * 256, bo = ks * (BN / 8) * 256;
        const uint64_t dah = smem_desc(a_hi + ao, 128, 256), dal = smem_desc(a_lo + ao, 128, 256);
        const uint64_t dbh = smem_desc(b_hi + bo, 128, 256), dbl = smem_desc(b_lo + bo, 128, 256);
        const uint32_t acc0 = (kt > 0 || ks > 0) ? 1u : 0u;
        mma_bf16(tmem, dah, dbh, idesc, acc0);
        mma_bf16(tmem, dah, dbl, idesc, 1u);
        mma_bf16(tmem, dal, dbh, idesc, 1u);
      }
      mma_commit(&bar_empty[st]);
      if (kt == ntiles - 1) mma_commit(&bar_done);
    }
    if (kt == ntiles - 1) committed_done = true;
    if (kt + 1 < ntiles) {
      advance();
      fetch();
    }
  }
  if (ntiles > 0 && !committed_done) {
    // aborted: track this CTA's issued MMAs on bar_done before freeing TMEM
    if (tid == 0) mma_commit(&bar_done);
    committed_done = true;
  }
  bool done_ok = true;
  if (ntiles > 0) done_ok = mbar_wait(&bar_done, 0);
  if (!ok || !done_ok || abort_sh) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
  } else {
    tc_fence_after();
    // epilogue: warp w owns D rows 32w .. 32w + 31 (TMEM lanes)
    const int drow = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
          "%10, %11, %12, %13, %14, %15}, [%16];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (drow < Mu) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int dcol = n0 + c0 + j;
          if (dcol >= Nu) break;
          const int gm = swap ? dcol : drow, gn = swap ? drow : dcol;
          float v = ntiles > 0 ? alpha * __uint_as_float(r[j]) : 0.f;
          if (it.Cin) v += beta * float(it.Cin[gm + (long long)gn * it.ldcin]);
          it.C[gm + (long long)gn * it.ldc] = TC(v);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(TMEM_COLS));
}

template <int BN, typename TC>
void launch_bn(const GemmItem<float, TC> *items, const GemmSeg<float> *segs, int nitems,
               int mu_max, int nu_max, bool trans, bool swap, float alpha, float beta,
               cudaStream_t s) {
  constexpr int STAGE_BYTES = 2 * BM * BK * 2 + 2 * BN * BK * 2;
  const size_t smem = (size_t)STAGES * STAGE_BYTES + 128;
  HODLR_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel<BN, TC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(nitems, cdiv(mu_max, BM), cdiv(nu_max, BN));
  tc_gemm_kernel<BN, TC><<<grid, kThreads, smem, s>>>(items, segs, alpha, beta, trans ? 1 : 0,
                                                      swap ? 1 : 0);
  HODLR_LAUNCH_CHECK();
}

}  // namespace

template <typename TC>
void launch_tc_gemm(const GemmItem<float, TC> *items, const GemmSeg<float> *segs, int nitems,
                    int max_m, int max_n, bool trans, float alpha, float beta, cudaStream_t s) {
  if (nitems <= 0 || max_m <= 0 || max_n <= 0) return;
  // put the wider side on the UMMA M = 128 side
  const bool swap = max_m < 128 && max_n > max_m;
  const int mu = swap ? max_n : max_m, nu = swap ? max_m : max_n;
  if (nu <= 64) launch_bn<64, TC>(items, segs, nitems, mu, nu, trans, swap, alpha, beta, s);
  else launch_bn<128, TC>(items, segs, nitems, mu, nu, trans, swap, alpha, beta, s);
}

int tc_error_flag(bool reset) {
  int h = 0;
  if (cudaMemcpyFromSymbol(&h, g_tc_error, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  if (reset && h) {
    int z = 0;
    cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int));
  }
  return h;
}

template void launch_tc_gemm<float>(const GemmItem<float, float> *, const GemmSeg<float> *, int,
                                    int, int, bool, float, float, cudaStream_t);

}  // namespace hodlr
