// tc_gemm.cu -- split-BF16 tensor-core GEMM engine (tcgen05, sm_100a).
//
// The mixed-precision path runs its GEMMs (leaf TRSM/trailing updates, the
// reduce V^T [d | u] and the broadcast d -= u eta) on the 5th-generation
// tensor cores.  FP32 operands are split as x = hi + lo with hi = bf16(x),
// lo = bf16(x - hi), and each product is accumulated in FP32 in tensor memory
// as  A_hi B_hi + A_hi B_lo + A_lo B_hi  (the lo*lo term, ~2^-16 relative, is
// dropped; FP64 iterative refinement recovers full accuracy).
//
// One persistent CTA per SM (17 warps) computes 128 x BN tiles of the items:
//   * two 4-warp producer groups (A tile, B tile) stage 32 K-values per row
//     and stage from global memory with cp.async, a few stages ahead, each
//     group cooperatively (whole 128-byte row runs or 512-byte column runs
//     per warp instruction); then every producer thread splits its own row
//     into hi/lo bf16 in the UMMA canonical K-major layout (8-row x 16-byte
//     core matrices, no swizzle);
//   * a 2- or 3-stage UMMA operand ring; one lane of the MMA warp issues the
//     MMAs (tcgen05.mma.cta_group::1.kind::f16, M = 128, N = BN, K = 16) and
//     tcgen05.commit arrives on the stage's mbarrier when the tensor cores are
//     done with it; producers wait on that barrier before reusing the stage;
//   * two accumulators live in TMEM (BN columns each, allocated per CTA); the
//     epilogue warps read one with tcgen05.ld (32 lanes per warp) and write
//     alpha * acc + beta * Cin to global memory while the next tile
//     accumulates into the other.
// The reduce's V^T X (M = r small, N wide) runs "swapped": the UMMA M side is
// the item's N and the result is written transposed.
// Every mbarrier wait is bounded; on timeout the kernel raises g_tc_error,
// waits (bounded) for its own MMAs, frees its TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "gemm_simt.cuh"
#include "tc_gemm.cuh"

namespace hodlr {

__device__ int g_tc_error = 0;
// Test hooks of the timeout path (hodlr_debug_tc_wait_hook): the bound of
// every mbarrier wait, and a one-shot request that the MMA issuer of CTA 0
// leave out the completion signal of its first tile, so that the epilogue's
// bounded wait for that tile runs out and the kernel takes its error exit.
__device__ long long g_tc_spin_limit = 1LL << 22;
__device__ int g_tc_skip_commit = 0;

namespace {

constexpr int BM = 128;    // UMMA M
// Operand split: hi = bf16(x), lo = bf16(x - hi) (kind::f16), each product
// accurate to ~2^-16 relative.  A TF32 split (kind::tf32, ~2^-21) was
// measured at N = 262144 (r = 64, m = 16): both need two FP64 refinement
// sweeps to reach 1e-12 (after one sweep 2.8e-11 with TF32, 9.6e-13 with
// plain FP32 FMA), so the cheaper BF16 split is used; its hi / lo pair also
// takes exactly the bytes of the FP32 value, so a stage is split in place.
constexpr int ELEM = 2;    // bytes per split operand element
constexpr int BK = 32;     // K per stage: 64 bytes of hi (and of lo) per operand row
constexpr int MMA_K = 16;  // K per tcgen05.mma kind::f16
// Bounded mbarrier waits: each try_wait may suspend the thread for up to
// kSuspendNs (it returns as soon as the phase completes), so waiting warps
// do not take issue slots from the working ones; g_tc_spin_limit tries
// (2^22 by default, a few seconds) bound a wait before the kernel gives up.
constexpr long long kSpinLimitDefault = 1LL << 22;
constexpr unsigned kSuspendNs = 1000;

__device__ inline uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ inline void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait for the completion of phase `parity`; false on timeout.
// `suspend` is the try_wait suspend-time hint in ns (0: poll).
__device__ inline bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit,
                                 uint32_t suspend = kSuspendNs) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(suspend)
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

// Instruction descriptor: kind::f16 with A = B = BF16, D = F32, both K-major.
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
// stage holding `rows` rows x BK k: [kstep][row/8][k-chunk][row%8][16 bytes].
__device__ inline uint32_t kmajor_off(int rows, int row, int kchunk_global) {
  const int ks = kchunk_global >> 1, kc = kchunk_global & 1;
  return (uint32_t)(ks * (rows / 8) * 256 + (row >> 3) * 256 + kc * 128 + (row & 7) * 16);
}

// Split 8 FP32 values into hi / lo bf16 and store one 16-byte chunk of each.
// Pairs go through the packed conversion: hi = bf16x2(x), lo = bf16x2(x - hi).
__device__ inline void split_store8(const float *v, unsigned char *hi, unsigned char *lo,
                                    uint32_t off) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const __nv_bfloat162 hb = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    const uint32_t hu = *reinterpret_cast<const uint32_t *>(&hb);
    const float h0 = __uint_as_float(hu << 16), h1 = __uint_as_float(hu & 0xffff0000u);
    const __nv_bfloat162 lb = __floats2bfloat162_rn(v[2 * q] - h0, v[2 * q + 1] - h1);
    h[q] = hu;
    l[q] = *reinterpret_cast<const uint32_t *>(&lb);
  }
  *reinterpret_cast<uint4 *>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4 *>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ inline void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Persistent, warp-specialized split-operand GEMM.
//   warps 0-7 (producers): two 4-warp groups stage the tiles with cp.async a
//     few stages ahead (cp.async.wait_group, then the group's named
//     barrier); thread p then splits row p of a tile into hi / lo in place,
//     in the UMMA K-major layout (full[s]: one arrival per thread that
//     splits, empty[s]: tcgen05.commit).  Either group 0 takes the A tile
//     and group 1 the B tile of every stage, or (prod_streams == 2) each
//     group takes both tiles of every other stage.
//   warp 8 lane 0 (MMA issuer): 3 MMAs per k-step into one of two TMEM
//     accumulators (tfull[a]: commit; tready[a]: one arrival per epilogue
//     thread once the buffer is drained and preloaded with the next tile's
//     scaled Cin).
//   warps 9-16 (epilogue): two warps per TMEM lane quarter, each owning one
//     row of the tile and half of its columns.  Tile j's C is staged by
//     cp.async while tile j - 1 computes, copied into the accumulator of
//     tile j before its MMAs (scaled by beta / alpha), and the drain writes
//     alpha * acc: C = alpha (A B + (beta / alpha) Cin).
constexpr int kEpiWarps = 8;  // two per TMEM lane quarter, each half of the columns
constexpr int kEpiThreads = kEpiWarps * 32;
constexpr int kProdWarps = 8;  // 4 for the A tile rows, 4 for the B tile rows
constexpr int kMmaWarp = kProdWarps;
constexpr int kEpiWarp0 = kProdWarps + 1;
constexpr int kWarps = kProdWarps + 1 + kEpiWarps;
constexpr int kThreadsP = kWarps * 32;
// One ring of stages, each the A tile (128 rows) and the B tile (BN rows) of
// BK k-values: the cp.async copies land there as FP32, and each producer
// thread then overwrites its row with the hi / lo bf16 split in the UMMA
// canonical layout (the same bytes), which the MMAs read.  Measured on this
// part: scattered 128-byte row runs read at 2.3 TB/s with 64 KB per SM in
// flight, 4.1 TB/s with 128 KB and 4.6 TB/s with 256 KB (a stage lands 3-5 us
// after its copies are issued under load), so the ring is as deep as the
// shared memory allows next to the C staging: 5 stages of 32 KB for
// 128-column tiles, 8 of 24 KB for 64-column ones.
template <int BN>
__host__ __device__ constexpr int stage_bytes() { return (128 + BN) * BK * 4; }
// C tile staging (launches with beta != 0 only)
template <int BN, bool CIN>
__host__ __device__ constexpr int cst_bytes() { return CIN ? (BN + 4) * 128 * 4 : 0; }
constexpr int kSmemPerCta = 232448;  // 227 KB opt-in shared memory per CTA
constexpr int kStaticSmem = 256;     // the kernel's barriers and flags
// A group refills the slot of its stage i - kRefillLag after handing stage i
// to the MMA warp (the MMAs of a stage complete ~0.2 us after their commit).
constexpr int kRefillLag = 1;
template <int BN, bool CIN>
__host__ __device__ constexpr int ring_depth() {
  return (kSmemPerCta - kStaticSmem - 128 - cst_bytes<BN, CIN>()) / stage_bytes<BN>();
}
// Independent copy / split loops per CTA: on this part one loop with a deep
// ring reads scattered 128-byte row runs at ~2.8 TB/s over the GPU whatever
// its depth (cp.async or TMA), two loops per SM at ~3.8-4.2 TB/s.  Two where
// the ring gives each at least 3 stages (all but 128-column tiles with C
// staging, which keep one loop over 5 stages); an odd last slot is unused.
template <int BN, bool CIN>
__host__ __device__ constexpr int prod_streams() {
  return ring_depth<BN, CIN>() / 2 >= 2 ? 2 : 1;
}
// refill lag of a group with DG ring slots: 1, or 0 where DG = 2 (the group
// then waits for the MMAs of the stage it has just handed over)
__host__ __device__ constexpr int refill_lag(int dg) { return dg >= 3 ? kRefillLag : 0; }
// ring slots in use: a multiple of the stream count
template <int BN, bool CIN>
__host__ __device__ constexpr int ring_slots() {
  return ring_depth<BN, CIN>() / prod_streams<BN, CIN>() * prod_streams<BN, CIN>();
}

__device__ inline void cpa4(void *dst, const void *src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(ok ? 4 : 0));
}
__device__ inline void cpa16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src));
}
__device__ inline void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Position in the flattened (tile, segment, k0) sequence of a CTA.
template <typename TC>
struct KPos {
  int t, seg, k0;
  int m0, n0, Mu, Nu;
  GemmItem<float, TC> it;
  GemmSeg<float> sg;
  bool valid;
};

// Stage one row of an M-contiguous operand (row `row`, its BK k-values ld
// apart) into `dst` (BK floats, the thread's own staging row) with 4-byte
// cp.async copies; consecutive lanes own consecutive rows, so each warp
// instruction reads 128 contiguous bytes.  Zero-filled outside the matrix.
// The row's 16-byte chunks are XOR-swizzled by `sw` (= row & 7) so that the
// 32 lanes reading their rows chunk by chunk hit distinct banks.
__device__ inline void cpa4_u(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)), "l"(src));
}
__device__ inline void stage_row_strided(float *dst, int sw, const float *base, long long ld,
                                         int row, int rows_valid, int k0, int K) {
  float *chunk[BK / 4];
#pragma unroll
  for (int g = 0; g < BK / 4; ++g) chunk[g] = dst + ((g ^ sw) << 2);
  const bool inrow = row < rows_valid;
  const float *p = base + row + (long long)k0 * ld;
  if (inrow && k0 + BK <= K) {
#pragma unroll
    for (int k = 0; k < BK; ++k) cpa4_u(chunk[k >> 2] + (k & 3), p + (long long)k * ld);
  } else {
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      const bool ok = inrow && k0 + k < K;
      cpa4(chunk[k >> 2] + (k & 3), ok ? p + (long long)k * ld : base, ok);
    }
  }
}

// Stage a K x rows column-major operand block (rows contiguous in memory) as
// a [BK][128] column tile, cooperatively: warp w of the 4-warp group copies
// k-columns w, w + 4, ...; lane l copies rows 4 l .. 4 l + 3 with one 16-byte
// copy when the block is aligned and fully inside the matrix.
__device__ inline void stage_cols(float *dst, int wg, int lane, const float *base, long long ld,
                                  int row0, int rows_valid, int k0, int K) {
  const int r = row0 + 4 * lane;
  const bool vec = ((reinterpret_cast<uintptr_t>(base) & 15) == 0) && ((ld & 3) == 0);
#pragma unroll
  for (int kk = 0; kk < BK / 4; ++kk) {
    const int k = wg + 4 * kk;
    float *d = dst + k * 128 + 4 * lane;
    const float *src = base + r + (long long)(k0 + k) * ld;
    const bool kin = k0 + k < K;
    if (vec && kin && r + 4 <= rows_valid) {
      cpa16(d, src);
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool ok = kin && r + u < rows_valid;
        cpa4(d + u, ok ? src + u : base, ok);
      }
    }
  }
}

// Stage NROWS K-contiguous operand rows (row r: base[(row0 + r) ld + k0 ..
// + BK)) into the group's staging region, cooperatively: thread t of the
// 4-warp group copies 16-byte chunk t % CPR of rows t / CPR, t / CPR +
// 128 / CPR, ... (CPR = BK / 4 chunks per row), so that one BF16-split warp
// instruction covers four whole 128-byte row runs (one L2 request each)
// instead of a 16-byte piece of 32 different rows.  Row r lands at dst + r BK
// with its chunks XOR-swizzled like stage_row_strided's, the layout that thread r
// reads back.  Zero-filled outside the matrix.
template <int NROWS>
__device__ inline void stage_rows_coop(float *dst, int t, const float *base, long long ld,
                                       int row0, int rows_valid, int k0, int K) {
  constexpr int CPR = BK / 4;
  constexpr int RPP = 128 / CPR;  // rows per pass of the group
  static_assert(NROWS % RPP == 0, "whole passes");
  const int c = t % CPR;
  const int kc = k0 + 4 * c;
  const bool vec = ((reinterpret_cast<uintptr_t>(base) & 15) == 0) && ((ld & 3) == 0);
  const bool kfull = kc + 4 <= K;
#pragma unroll
  for (int i = 0; i < NROWS / RPP; ++i) {
    const int r = t / CPR + RPP * i;
    const int gr = row0 + r;
    const int sw = r & 7;
    float *d = dst + r * BK + ((c ^ sw) << 2);
    const float *src = base + (long long)gr * ld + kc;
    if (vec && kfull && gr < rows_valid) {
      cpa16(d, src);
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool ok = gr < rows_valid && kc + u < K;
        cpa4(d + u, ok ? src + u : base, ok);
      }
    }
  }
}

template <int BN, bool SWAP, typename TC, bool CIN>
__global__ void __launch_bounds__(kThreadsP, 1)
    tc_gemm_persistent(const GemmItem<float, TC> *__restrict__ items,
                       const GemmSeg<float> *__restrict__ segs, int nitems, int mtiles,
                       int ntn, float alpha, float beta, int trans, unsigned suspend) {
  static_assert(sizeof(TC) == 4, "the engine writes FP32 results");
  constexpr bool swap = SWAP;
  constexpr int A_BYTES = BM * BK * ELEM;  // one of hi / lo
  constexpr int B_BYTES = BN * BK * ELEM;
  constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static_assert(STAGE_BYTES == stage_bytes<BN>(), "the split fills the FP32 stage exactly");
  constexpr int kStagesP = ring_slots<BN, CIN>();
  static_assert(kStagesP >= 3, "at least one stage in flight while one is split");
  constexpr int TMEM_COLS = 2 * BN;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *ring = smem;
  float *cst = reinterpret_cast<float *>(smem + kStagesP * STAGE_BYTES);  // C tile, 128 x (BN + 4)
  __shared__ __align__(8) uint64_t full[kStagesP], empty[kStagesP], tfull[2], tready[2], fin;
  __shared__ uint32_t tmem_sh;
  __shared__ volatile int abort_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int total = nitems * mtiles * ntn;
  const long long spin_limit = g_tc_spin_limit > 0 ? g_tc_spin_limit : kSpinLimitDefault;

  if (tid == 0) {
    for (int s = 0; s < kStagesP; ++s) {
      mbar_init(&full[s], kProdWarps * 32 / prod_streams<BN, CIN>());
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tready[a], kEpiThreads);
    }
    mbar_init(&fin, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;

  // t / d for t < 2^24 through a float reciprocal, corrected to the exact quotient
  const int mn = mtiles * ntn;
  const float inv_mn = 1.0f / float(mn), inv_n = 1.0f / float(ntn);
  auto qdiv = [](int t, int d, float inv) {
    int q = __float2int_rz(float(t) * inv);
    if (q * d > t) --q;
    else if ((q + 1) * d <= t) ++q;
    return q;
  };
  auto decode = [&](int t, GemmItem<float, TC> &it, int &m0, int &n0, int &Mu, int &Nu) {
    const int item = qdiv(t, mn, inv_mn);
    const int rem = t - item * mn;
    const int mt = qdiv(rem, ntn, inv_n);
    m0 = mt * BM;
    n0 = (rem - mt * ntn) * BN;
    it = items[item];
    Mu = swap ? it.N : it.M;
    Nu = swap ? it.M : it.N;
    return m0 < Mu && n0 < Nu;
  };
  auto kstages = [&](const GemmItem<float, TC> &it) {
    int n = 0;
    for (int s = it.seg_begin; s < it.seg_begin + it.seg_count; ++s) n += (segs[s].K + BK - 1) / BK;
    return n;
  };
  // first / next k-stage of the CTA's flattened sequence (skips empty tiles
  // and zero-length segments)
  auto first_in_tile = [&](KPos<TC> &ps) {
    for (; ps.t < total; ps.t += gridDim.x) {
      if (!decode(ps.t, ps.it, ps.m0, ps.n0, ps.Mu, ps.Nu)) continue;
      for (ps.seg = ps.it.seg_begin; ps.seg < ps.it.seg_begin + ps.it.seg_count; ++ps.seg) {
        ps.sg = segs[ps.seg];
        if (ps.sg.K > 0) { ps.k0 = 0; ps.valid = true; return; }
      }
    }
    ps.valid = false;
  };
  auto next = [&](KPos<TC> &ps) {
    ps.k0 += BK;
    if (ps.k0 < ps.sg.K) return;
    for (++ps.seg; ps.seg < ps.it.seg_begin + ps.it.seg_count; ++ps.seg) {
      ps.sg = segs[ps.seg];
      if (ps.sg.K > 0) { ps.k0 = 0; return; }
    }
    ps.t += gridDim.x;
    first_in_tile(ps);
  };

  if (warp < kProdWarps) {
    // ------------------------------------------------------------ producers
    // NS == 1: group 0 (warps 0-3) stages and splits the A tile, group 1
    // (warps 4-7) the B tile of every stage.  NS == 2: group g stages and
    // splits both tiles of the stages s = g (mod 2), in its own half of the
    // ring (the slots of parity g): two independent copy / split loops per
    // SM.  Thread p owns row p of each tile it splits (rows p >= BN of the B
    // tile do not exist).
    constexpr int NS = prod_streams<BN, CIN>();
    const int grp = warp >> 2;
    const bool doA = NS == 2 || grp == 0;
    const bool doB = NS == 2 || grp == 1;
    const int p = tid & 127;
    const int sw = p & 7;
    KPos<TC> iss, con;
    iss.t = con.t = blockIdx.x;
    first_in_tile(iss);
    first_in_tile(con);
    auto adv = [&](KPos<TC> &ps) {
#pragma unroll
      for (int i = 0; i < NS; ++i)
        if (ps.valid) next(ps);
    };
    if (NS == 2 && grp == 1) {  // group 1 starts at stage 1
      if (iss.valid) next(iss);
      if (con.valid) next(con);
    }
    // Each group stages cooperatively and synchronizes on its own named
    // barrier before reading a landed stage and before overwriting it with
    // the split: the M-contiguous A tile (A when !trans) column-wise
    // (stage_cols), K-contiguous rows 8 lanes per 128-byte run
    // (stage_rows_coop).  Only the swapped items' M-contiguous operand (at
    // most BN = 64 rows, one 4-byte column element per thread and k, i.e.
    // 128 contiguous bytes per warp instruction) is staged by each row's
    // owner.
    const bool colmode = !swap && trans == 0;  // of the A tile
    const int gbar = 2 + grp;                  // named barrier of this producer group
    auto group_sync = [&]() { asm volatile("bar.sync %0, 128;\n" ::"r"(gbar) : "memory"); };
    // ring slot `slot`: the A tile's FP32 rows at its start, then the same
    // bytes as A_hi | A_lo; the B tile's (BN rows) after them, then B_hi | B_lo
    auto a_part = [&](int slot) { return ring + slot * STAGE_BYTES; };
    auto b_part = [&](int slot) { return ring + slot * STAGE_BYTES + 2 * A_BYTES; };
    auto issue = [&](KPos<TC> &ps, int slot) {
      if (ps.valid) {
        const GemmSeg<float> &sg = ps.sg;
        if (doA) {
          float *region = reinterpret_cast<float *>(a_part(slot));
          if (!swap) {
            if (colmode) stage_cols(region, warp & 3, lane, sg.A, sg.lda, ps.m0, ps.it.M, ps.k0, sg.K);
            else stage_rows_coop<128>(region, p, sg.A, sg.lda, ps.m0, ps.it.M, ps.k0, sg.K);
          } else {
            stage_rows_coop<128>(region, p, sg.B, sg.ldb, ps.m0, ps.it.N, ps.k0, sg.K);
          }
        }
        if (doB) {
          float *region = reinterpret_cast<float *>(b_part(slot));
          if (!swap) {
            stage_rows_coop<BN>(region, p, sg.B, sg.ldb, ps.n0, ps.it.N, ps.k0, sg.K);
          } else if (trans != 0) {
            stage_rows_coop<BN>(region, p, sg.A, sg.lda, ps.n0, ps.it.M, ps.k0, sg.K);
          } else if (p < BN) {
            stage_row_strided(region + p * BK, sw, sg.A, sg.lda, ps.n0 + p, ps.it.M, ps.k0, sg.K);
          }
        }
        adv(ps);
      }
      cpa_commit();
    };
    // exit decision: uniform within a group that shares barriers (a thread
    // whose wait timed out raises abort_sh and the next vote ends the group)
    auto group_vote_or = [&](bool pr) -> bool {
      uint32_t r;
      asm volatile(
          "{\n\t.reg .pred pi, po;\n\t"
          "setp.ne.u32 pi, %1, 0;\n\t"
          "bar.red.or.pred po, %2, 128, pi;\n\t"
          "selp.u32 %0, 1, 0, po;\n\t}\n"
          : "=r"(r)
          : "r"((uint32_t)pr), "r"(gbar)
          : "memory");
      return r != 0;
    };
    // this thread's FP32 row (swizzled 16-byte chunks) or, for the
    // column-staged A tile, column entries
    auto read_row = [&](const unsigned char *part, float *v) {
      const float *row = reinterpret_cast<const float *>(part) + p * BK;
#pragma unroll
      for (int q = 0; q < BK / 4; ++q) {
        const float4 x = reinterpret_cast<const float4 *>(row)[q ^ sw];
        v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
      }
    };
    auto read_a = [&](const unsigned char *part, float *v) {
      if (colmode) {
        const float *col = reinterpret_cast<const float *>(part);
#pragma unroll
        for (int k = 0; k < BK; ++k) v[k] = col[k * 128 + p];
      } else {
        read_row(part, v);
      }
    };
    auto split_a = [&](unsigned char *part, const float *v) {
#pragma unroll
      for (int c = 0; c < 4; ++c) split_store8(v + 8 * c, part, part + A_BYTES, kmajor_off(BM, p, c));
    };
    auto split_b = [&](unsigned char *part, const float *v) {
#pragma unroll
      for (int c = 0; c < 4; ++c) split_store8(v + 8 * c, part, part + B_BYTES, kmajor_off(BN, p, c));
    };
    // This group's stages use DG = D / NS ring slots (slot of local stage i:
    // g0 + NS (i % DG)).  Local stages 0 .. DG - L - 1 are issued up front;
    // iteration i waits for stage i, splits it in place, hands it to the MMA
    // warp (full), then refills the slot of local stage i - L -- freed by its
    // MMAs (empty) -- with local stage i + DG - L, so DG - L - 1 stages stay
    // in flight while one is split.  con advances alike in every thread
    // (timeouts included), so the loop condition is uniform across the group.
    constexpr int D = kStagesP;
    static_assert(D % NS == 0, "whole slots per group");
    constexpr int DG = D / NS;
    constexpr int L = refill_lag(DG);
    static_assert(DG - L - 1 >= 1, "a stage in flight while one is split");
    const int g0 = NS == 2 ? grp : 0;
    for (int i = 0; i < DG - L; ++i) issue(iss, g0 + NS * i);
    int li = 0;             // local slot of stage i
    int rli = (DG - L) % DG;       // local slot refilled in iteration i: the one of stage i - L
    uint32_t rphase = L > 0 ? 1 : 0;  // parity of the empty phase that frees it (fresh: 1)
    while (con.valid) {
      cpa_wait<DG - L - 1>();  // this thread's copies of stage i have landed
      group_sync();            // ... and the whole group's
      const int slot = g0 + NS * li;
      float v[BK];
      if (doA) read_a(a_part(slot), v);
      else if (p < BN) read_row(b_part(slot), v);
      // every thread has read its FP32 row before the part is overwritten;
      // the same barrier makes the group's exit decision
      if (group_vote_or(abort_sh)) break;
      if (doA) split_a(a_part(slot), v);
      else if (p < BN) split_b(b_part(slot), v);
      if (NS == 2) {  // then the B tile of the same stage
        if (p < BN) read_row(b_part(slot), v);
        group_sync();
        if (p < BN) split_b(b_part(slot), v);
      }
      fence_proxy_async();
      mbar_arrive(&full[slot]);
      if (mbar_wait(&empty[g0 + NS * rli], rphase, spin_limit, suspend)) {
        issue(iss, g0 + NS * rli);
      } else {
        abort_sh = 1;  // the group leaves together at the next vote
        cpa_commit();  // keep one copy group per stage
      }
      if (++rli == DG) { rli = 0; rphase ^= 1; }
      if (++li == DG) li = 0;
      adv(con);
    }
    cpa_wait<0>();
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t idesc = instr_desc(BM, BN);
      int stage = 0, acc = 0;
      uint32_t phase = 0, aphase = 0;
      // test hook: leave out the first tile's completion signal (one launch)
      bool skip_commit = blockIdx.x == 0 && atomicExch(&g_tc_skip_commit, 0) != 0;
      for (int t = blockIdx.x; t < total && !abort_sh; t += gridDim.x) {
        GemmItem<float, TC> it;
        int m0, n0, Mu, Nu;
        if (!decode(t, it, m0, n0, Mu, Nu)) continue;
        // the epilogue has drained this accumulator and preloaded it with
        // (beta / alpha) Cin when the item has one
        if (!mbar_wait(&tready[acc], aphase, spin_limit, suspend)) { abort_sh = 1; break; }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * BN);
        const int nst = kstages(it);
        const uint32_t pre = (CIN && it.Cin != nullptr && beta != 0.f) ? 1u : 0u;
        for (int ks_all = 0; ks_all < nst; ++ks_all) {
          if (!mbar_wait(&full[stage], phase, spin_limit, suspend)) { abort_sh = 1; break; }
          tc_fence_after();
          const uint32_t a_hi = smem_u32(ring + stage * STAGE_BYTES), a_lo = a_hi + A_BYTES;
          const uint32_t b_hi = a_hi + 2 * A_BYTES, b_lo = b_hi + B_BYTES;
#pragma unroll
          for (int ks = 0; ks < BK / MMA_K; ++ks) {
            const uint32_t ao = ks * (BM / 8) * 256, bo = ks * (BN / 8) * 256;
            const uint64_t dah = smem_desc(a_hi + ao, 128, 256), dal = smem_desc(a_lo + ao, 128, 256);
            const uint64_t dbh = smem_desc(b_hi + bo, 128, 256), dbl = smem_desc(b_lo + bo, 128, 256);
            mma_bf16(d, dah, dbh, idesc, (ks_all > 0 || ks > 0) ? 1u : pre);
            mma_bf16(d, dah, dbl, idesc, 1u);
            mma_bf16(d, dal, dbh, idesc, 1u);
          }
          mma_commit(&empty[stage]);
          if (++stage == kStagesP) { stage = 0; phase ^= 1; }
        }
        if (abort_sh) break;
        if (skip_commit) skip_commit = false;
        else mma_commit(&tfull[acc]);
        if (++acc == 2) { acc = 0; aphase ^= 1; }
      }
      mma_commit(&fin);  // all MMAs of this CTA complete before TMEM is freed
      if (!mbar_wait(&fin, 0, spin_limit, suspend)) abort_sh = 1;
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;        // TMEM lane quarter of this warp
    const int rl = q * 32 + lane;  // row of the tile owned by this thread
    const int ew = warp - kEpiWarp0;  // epilogue warp 0..7
    const int half = ew >> 2;      // columns [half * BN / 2, (half + 1) * BN / 2)
    const int cbeg = half * (BN / 2), cend = cbeg + BN / 2;
    int acc = 0;
    uint32_t aphase = 0;
    // Cin staging.  Non-swapped tiles: cst[j * 128 + row] (column j of the
    // tile, filled a whole column per warp instruction with 16-byte copies).
    // Swapped tiles: cst[row * CSTR + j] (row = item column, contiguous in
    // memory along j, filled by the row's owner with 16-byte copies).
    constexpr int CSTR = BN + 4;
    auto issue_c = [&](const GemmItem<float, TC> &it, int m0, int n0, int Mu, int Nu) {
      if (CIN && it.Cin != nullptr) {
        const float *cin = reinterpret_cast<const float *>(it.Cin);
        const long long ld = it.ldcin;
        const bool vec = ((reinterpret_cast<uintptr_t>(cin) & 15) == 0) && ((ld & 3) == 0);
        if (!SWAP) {
          // lane covers rows m0 + 4 lane .. + 3 of column n0 + j
          const int r4 = m0 + 4 * lane;
          for (int j = ew; j < BN; j += kEpiWarps) {
            const int dcol = n0 + j;
            float *dst = cst + j * 128 + 4 * lane;
            const float *src = cin + r4 + (long long)dcol * ld;
            if (vec && dcol < Nu && r4 + 4 <= Mu) {
              cpa16(dst, src);
            } else {
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const bool ok = dcol < Nu && r4 + u < Mu;
                cpa4(dst + u, ok ? src + u : cin, ok);
              }
            }
          }
        } else {
          // this thread's item column gn = m0 + rl, item rows n0 .. n0 + BN
          const int gn = m0 + rl;
          float *dst = cst + rl * CSTR;
          const float *src = cin + n0 + (long long)gn * ld;
          const bool rowok = gn < Mu;
          for (int j = cbeg; j < cend; j += 4) {
            if (vec && rowok && n0 + j + 4 <= Nu) {
              cpa16(dst + j, src + j);
            } else {
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const bool ok = rowok && n0 + j + u < Nu;
                cpa4(dst + j + u, ok ? src + j + u : cin, ok);
              }
            }
          }
        }
      }
      cpa_commit();
    };
    auto epi_sync = [&]() { asm volatile("bar.sync 1, %0;\n" ::"n"(kEpiThreads) : "memory"); };
    // barrier of the epilogue threads returning the OR of `p` (uniform exit decisions)
    auto epi_vote_or = [&](bool p) -> bool {
      uint32_t r;
      asm volatile(
          "{\n\t.reg .pred pi, po;\n\t"
          "setp.ne.u32 pi, %1, 0;\n\t"
          "bar.red.or.pred po, 1, %2, pi;\n\t"
          "selp.u32 %0, 1, 0, po;\n\t}\n"
          : "=r"(r)
          : "r"((uint32_t)p), "n"(kEpiThreads)
          : "memory");
      return r != 0;
    };
    const float cscale = beta / alpha;  // alpha != 0 (launch_tc_gemm routes alpha = 0 away)
    // The epilogue's tile sequence: tile j uses accumulator j & 1.  After
    // tile j is drained, its buffer is preloaded with tile j + 2's
    // (beta / alpha) Cin from the staging buffer (filled by cp.async while
    // tile j + 1 was computed) and released to the MMA issuer, which then
    // accumulates alpha^{-1}-scaled products onto it; the drain multiplies by
    // alpha.
    struct Tile {
      GemmItem<float, TC> it;
      int m0, n0, Mu, Nu;
      bool valid;
    };
    int tnext = blockIdx.x;
    auto fetch = [&](Tile &T) {
      T.valid = false;
      for (; tnext < total; tnext += gridDim.x)
        if (decode(tnext, T.it, T.m0, T.n0, T.Mu, T.Nu)) {
          T.valid = true;
          tnext += gridDim.x;
          return;
        }
    };
    // staged Cin (landed, visible to all epilogue threads) -> TMEM buffer b
    auto preload = [&](const Tile &T, int b) {
      if constexpr (!CIN) return;
      if (!(T.it.Cin != nullptr && beta != 0.f)) return;
#pragma unroll 1
      for (int c0 = cbeg; c0 < cend; c0 += 16) {
        uint32_t r[16];
        if (!SWAP) {
          const float *cs = cst + c0 * 128 + rl;
#pragma unroll
          for (int j = 0; j < 16; ++j) r[j] = __float_as_uint(cscale * cs[j * 128]);
        } else {
          const float *cs = cst + rl * CSTR + c0;
#pragma unroll
          for (int j = 0; j < 16; j += 4) {
            const float4 c4 = *reinterpret_cast<const float4 *>(cs + j);
            r[j] = __float_as_uint(cscale * c4.x);
            r[j + 1] = __float_as_uint(cscale * c4.y);
            r[j + 2] = __float_as_uint(cscale * c4.z);
            r[j + 3] = __float_as_uint(cscale * c4.w);
          }
        }
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + c0);
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15, %16};\n" ::"r"(taddr),
            "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
            "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]),
            "r"(r[14]), "r"(r[15]));
      }
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
    };
    auto release = [&](int b) {
      tc_fence_before();
      mbar_arrive(&tready[b]);
    };
    Tile cur, n1, n2;
    fetch(cur);
    fetch(n1);
    fetch(n2);
    // prologue: the first two tiles' buffers (uniform across the epilogue threads)
    if (cur.valid) {
      issue_c(cur.it, cur.m0, cur.n0, cur.Mu, cur.Nu);
      cpa_wait<0>();
      epi_sync();
      preload(cur, 0);
      epi_sync();  // staging free again
      release(0);
    }
    if (n1.valid) {
      issue_c(n1.it, n1.m0, n1.n0, n1.Mu, n1.Nu);
      cpa_wait<0>();
      epi_sync();
      preload(n1, 1);
      epi_sync();
      release(1);
    }
    if (n2.valid) issue_c(n2.it, n2.m0, n2.n0, n2.Mu, n2.Nu);
    else cpa_commit();
    while (cur.valid) {  // the tile sequence is uniform across the epilogue threads
      const GemmItem<float, TC> &it = cur.it;
      const int m0 = cur.m0, n0 = cur.n0, Mu = cur.Mu, Nu = cur.Nu;
      const bool live = kstages(it) > 0 || (CIN && it.Cin != nullptr && beta != 0.f);
      const bool ok = mbar_wait(&tfull[acc], aphase, spin_limit, suspend);
      cpa_wait<0>();  // tile j + 2's Cin staged by this thread
      // one barrier: every thread's copies visible, one exit decision for all
      if (epi_vote_or(!ok || abort_sh)) {
        if (!ok) abort_sh = 1;
        break;
      }
      tc_fence_after();
      float *C = reinterpret_cast<float *>(it.C);
      const long long ldc = it.ldc;
      const float a_eff = live ? alpha : 0.f;
#pragma unroll 1
      for (int c0 = cbeg; c0 < cend && n0 + c0 < Nu; c0 += 16) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
              "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        const int ncols = min(16, Nu - n0 - c0);
        if (!SWAP) {
          const int drow = m0 + rl;
          if (drow < Mu) {
            float *cp = C + drow + (long long)(n0 + c0) * ldc;
#pragma unroll
            for (int j = 0; j < 16; ++j)
              if (j < ncols) cp[(long long)j * ldc] = a_eff * __uint_as_float(r[j]);
          }
        } else {
          const int gn = m0 + rl;
          if (gn < Mu) {
            float *cp = C + (n0 + c0) + (long long)gn * ldc;
            if (ncols == 16 && (reinterpret_cast<uintptr_t>(cp) & 15) == 0) {
#pragma unroll
              for (int j = 0; j < 16; j += 4)
                *reinterpret_cast<float4 *>(cp + j) =
                    make_float4(a_eff * __uint_as_float(r[j]), a_eff * __uint_as_float(r[j + 1]),
                                a_eff * __uint_as_float(r[j + 2]), a_eff * __uint_as_float(r[j + 3]));
            } else {
#pragma unroll
              for (int j = 0; j < 16; ++j)
                if (j < ncols) cp[j] = a_eff * __uint_as_float(r[j]);
            }
          }
        }
      }
      // buffer `acc` now belongs to tile j + 2: preload its Cin and release it
      if (n2.valid) preload(n2, acc);
      epi_sync();  // staging free for tile j + 3
      release(acc);
      if (++acc == 2) { acc = 0; aphase ^= 1; }
      cur = n1;
      n1 = n2;
      fetch(n2);
      if (n2.valid) issue_c(n2.it, n2.m0, n2.n0, n2.Mu, n2.Nu);
      else cpa_commit();
    }
    cpa_wait<0>();
  }
  tc_fence_before();
  __syncthreads();
  if (abort_sh && tid == 0) atomicExch(&g_tc_error, 1);
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(TMEM_COLS));
}

template <int BN, bool SWAP, typename TC, bool CIN>
void launch_bn(const GemmItem<float, TC> *items, const GemmSeg<float> *segs, int nitems,
               int mu_max, int nu_max, bool trans, float alpha, float beta, cudaStream_t s) {
  const size_t smem = (size_t)ring_slots<BN, CIN>() * stage_bytes<BN>() + cst_bytes<BN, CIN>() + 128;
  raise_smem_limit(reinterpret_cast<const void *>(tc_gemm_persistent<BN, SWAP, TC, CIN>), smem);
  const int mt = cdiv(mu_max, BM), nt = cdiv(nu_max, BN);
  const long long total = (long long)nitems * mt * nt;
  int sms = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
  }
  const int grid = (int)std::min<long long>(total, sms);
  tc_gemm_persistent<BN, SWAP, TC, CIN><<<grid, kThreadsP, smem, s>>>(
      items, segs, nitems, mt, nt, alpha, beta, trans ? 1 : 0, kSuspendNs);
  HODLR_LAUNCH_CHECK();
}

// tile width by the UMMA N side, C staging only where beta != 0
template <bool SWAP, typename TC>
void launch_sw(const GemmItem<float, TC> *items, const GemmSeg<float> *segs, int nitems, int mu,
               int nu, bool trans, float alpha, float beta, cudaStream_t s) {
  if (beta != 0.f) {
    if (nu <= 64) launch_bn<64, SWAP, TC, true>(items, segs, nitems, mu, nu, trans, alpha, beta, s);
    else launch_bn<128, SWAP, TC, true>(items, segs, nitems, mu, nu, trans, alpha, beta, s);
  } else {
    if (nu <= 64) launch_bn<64, SWAP, TC, false>(items, segs, nitems, mu, nu, trans, alpha, beta, s);
    else launch_bn<128, SWAP, TC, false>(items, segs, nitems, mu, nu, trans, alpha, beta, s);
  }
}

}  // namespace

template <typename TC>
void launch_tc_gemm(const GemmItem<float, TC> *items, const GemmSeg<float> *segs, int nitems,
                    int max_m, int max_n, bool trans, float alpha, float beta, cudaStream_t s) {
  if (nitems <= 0 || max_m <= 0 || max_n <= 0) return;
  if (alpha == 0.f) {
    // C = beta Cin: the engine folds Cin into the accumulator as (beta / alpha) Cin
    launch_gemm_items<float, float, float>(reinterpret_cast<const GemmItem<float, float> *>(items),
                                           segs, nitems, max_m, max_n, trans, alpha, beta, s,
                                           false);
    return;
  }
  // put the wider side on the UMMA M = 128 side
  const bool swap = max_m < 128 && max_n > max_m;
  const int mu = swap ? max_n : max_m, nu = swap ? max_m : max_n;
  if (swap) {
    launch_sw<true, TC>(items, segs, nitems, mu, nu, trans, alpha, beta, s);
  } else {
    launch_sw<false, TC>(items, segs, nitems, mu, nu, trans, alpha, beta, s);
  }
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

void tc_set_wait_hook(long long polls, int skip_one_commit) {
  const long long lim = polls > 0 ? polls : kSpinLimitDefault;
  const int skip = skip_one_commit ? 1 : 0;
  HODLR_CUDA_TRY(cudaMemcpyToSymbol(g_tc_spin_limit, &lim, sizeof(lim)));
  HODLR_CUDA_TRY(cudaMemcpyToSymbol(g_tc_skip_commit, &skip, sizeof(skip)));
}

template void launch_tc_gemm<float>(const GemmItem<float, float> *, const GemmSeg<float> *, int,
                                    int, int, bool, float, float, cudaStream_t);

}  // namespace hodlr
