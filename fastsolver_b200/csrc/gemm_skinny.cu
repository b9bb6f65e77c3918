// gemm_skinny.cu -- batched GEMM items with at most 32 columns (the m
// right-hand sides): the refinement sweeps' reduce / broadcast and the FP64
// HODLR matvec (gemm_simt.cu routes them here).
//
// These products stream a tall operand (V, U or D, up to a few GB per
// launch) against a small one, so they are bound by HBM bandwidth; both
// kernels keep every operand tile in flight with a 3-stage cp.async ring
// (16-byte copies where the addresses allow) and compute from shared memory.
//
//   skinny_nn2: C (M x N) = beta Cin + alpha sum_s A_s B_s, A_s M x K column-
//               major.  CTA = 512 rows of one item, thread = 2 rows, 2 x NC
//               accumulators; per K tile the A tile (KT x 512) and the B tile
//               (KT x NC) land in shared memory.
//   skinny_tn2: C (M x N) = beta Cin + alpha sum_s A_s^T B_s, A_s K x M.
//               CTA (128 threads) = 64 x 16 block of C of one item over all
//               of K; thread = rows (m, m + 32) x 4 columns, the A and B tiles
//               stored k-contiguous so each thread reads 16-byte vectors along k.
#include <algorithm>

#include "common.cuh"
#include "gemm_skinny.cuh"
#include "skinny_units.cuh"

namespace hodlr {

namespace {

using namespace sk;
constexpr int kSkThreads = 256;

// ---------------------------------------------------------------- NN (rows)
// FP32 C (M x N <= NC) = beta Cin + alpha sum_s A_s B_s with one row per
// thread: A is read straight from global memory (a warp reads 32 consecutive
// rows of one column: 128 bytes), 32 (16 when NC = 32) k-values in flight
// per thread, while the matching block of B sits in shared memory.  Small CTAs (128 rows)
// and no A staging let many CTAs share an SM, which keeps enough loads in
// flight for the short-K products of the refinement sweeps (K = r).
// The CTAs (as many as are resident: three per SM at the kernel's 168
// registers) take the units (item, 128-row block) u = blockIdx.x,
// blockIdx.x + gridDim.x, ...: at N = 262144 the root's m-column broadcast
// has 2048 units, which as one CTA each ran in 4.6 waves of short CTAs.
template <int NC>
__global__ void __launch_bounds__(kRowThreads)
    skinny_nn_rows_kernel(const GemmItem<float, float> *__restrict__ items,
                          const GemmSeg<float> *__restrict__ segs, float alpha, float beta,
                          int nunits, int rbn) {
  __shared__ __align__(16) float Bs[nn_rows_kc<NC>() * NC];
  for (int u = blockIdx.x; u < nunits; u += gridDim.x)
    nn_rows_unit<NC>(items, segs, alpha, beta, u / rbn, u % rbn, Bs);
}

// ---------------------------------------------------------------- NN
// CTA = 512 rows of one item, thread = rows (r, r + 256), 2 x NC accumulators,
// so every broadcast read of B feeds two rows.
constexpr int kNNRows = 2 * kSkThreads;
template <typename T>
__host__ __device__ constexpr int nn_kt() { return sizeof(T) == 4 ? 16 : 8; }

// ring depth: FP64 runs one CTA per SM (register bound) and keeps five tiles
// in flight; FP32 two CTAs per SM with two each
template <typename T>
__host__ __device__ constexpr int nn_stages() { return sizeof(T) == 4 ? 3 : 6; }

template <typename T, int NC>
__global__ void __launch_bounds__(kSkThreads)
    skinny_nn2_kernel(const GemmItem<T, T> *__restrict__ items, const GemmSeg<T> *__restrict__ segs,
                      T alpha, T beta) {
  constexpr int KT = nn_kt<T>();
  constexpr int STG = nn_stages<T>();
  constexpr int ROWS = kNNRows;
  constexpr int VW = Vec<T>::W;
  using V = typename Vec<T>::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *As = reinterpret_cast<T *>(smem_raw);             // [stage][KT][ROWS]
  T *Bs = As + (size_t)STG * KT * ROWS;          // [stage][KT][NC]
  const GemmItem<T, T> it = items[blockIdx.x];
  const int row0 = blockIdx.y * ROWS;
  if (row0 >= it.M) return;
  const int tid = threadIdx.x;
  const int N = it.N;

  auto load = [&](const TileIter<T> &p, int st) {
    if (p.valid) {
      const GemmSeg<T> &sg = p.sg;
      T *a = As + (size_t)st * KT * ROWS;
      T *b = Bs + (size_t)st * KT * NC;
      const T *abase = sg.A + row0 + (long long)p.k0 * sg.lda;
      const bool vec = ((reinterpret_cast<uintptr_t>(abase) & 15) == 0) && ((sg.lda % VW) == 0);
      if (vec) {
        for (int e = tid; e < KT * (ROWS / VW); e += kSkThreads) {
          const int k = e / (ROWS / VW), rv = e % (ROWS / VW);
          const int r = row0 + rv * VW;
          const bool kin = p.k0 + k < sg.K;
          const T *src = abase + rv * VW + (long long)k * sg.lda;
          if (kin && r + VW <= it.M) {
            cpa(a + k * ROWS + rv * VW, src, 16, true);
          } else {
#pragma unroll
            for (int u = 0; u < VW; ++u) {
              const bool ok = kin && r + u < it.M;
              cpa(a + k * ROWS + rv * VW + u, ok ? src + u : sg.A, sizeof(T), ok);
            }
          }
        }
      } else {
        for (int e = tid; e < KT * ROWS; e += kSkThreads) {
          const int k = e / ROWS, rr = e % ROWS;
          const bool ok = (p.k0 + k < sg.K) && row0 + rr < it.M;
          cpa(a + k * ROWS + rr, ok ? abase + rr + (long long)k * sg.lda : sg.A, sizeof(T), ok);
        }
      }
      for (int e = tid; e < KT * NC; e += kSkThreads) {
        const int k = e % KT, n = e / KT;
        const bool ok = (p.k0 + k < sg.K) && n < N;
        cpa(b + k * NC + n, ok ? sg.B + (p.k0 + k) + (long long)n * sg.ldb : sg.B, sizeof(T), ok);
      }
    }
    cpa_commit();
  };

  T acc0[NC], acc1[NC];
#pragma unroll
  for (int n = 0; n < NC; ++n) { acc0[n] = T(0); acc1[n] = T(0); }
  TileIter<T> ld, cp;
  ld.init(segs, it.seg_begin, it.seg_count);
  cp = ld;
#pragma unroll
  for (int i = 0; i < STG - 1; ++i) {
    load(ld, i);
    if (ld.valid) ld.next(KT);
  }
  int st = 0, lst = STG - 1;
  while (cp.valid) {
    load(ld, lst);
    if (ld.valid) ld.next(KT);
    lst = (lst + 1) % STG;
    cpa_wait<STG - 1>();
    __syncthreads();
    const T *a = As + (size_t)st * KT * ROWS + tid;
    const T *b = Bs + (size_t)st * KT * NC;
#pragma unroll
    for (int k = 0; k < KT; ++k) {
      const T a0 = a[k * ROWS], a1 = a[k * ROWS + kSkThreads];
#pragma unroll
      for (int n = 0; n < NC; n += VW) {
        const V bv = *reinterpret_cast<const V *>(b + k * NC + n);
        const T *bp = reinterpret_cast<const T *>(&bv);
#pragma unroll
        for (int u = 0; u < VW; ++u) {
          acc0[n + u] += a0 * bp[u];
          acc1[n + u] += a1 * bp[u];
        }
      }
    }
    __syncthreads();  // stage st is refilled STG - 1 tiles later
    st = (st + 1) % STG;
    cp.next(KT);
  }
  cpa_wait<0>();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int row = row0 + tid + h * kSkThreads;
    if (row < it.M) {
      static_assert(NC % 8 == 0, "whole column groups");
      // per 8 columns: their Cin values before their stores (C may alias
      // Cin, so a load after a store would wait for it)
#pragma unroll
      for (int n8 = 0; n8 < NC; n8 += 8) {
        T cin[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
          cin[u] = (it.Cin && n8 + u < N) ? it.Cin[row + (long long)(n8 + u) * it.ldcin] : T(0);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int n = n8 + u;
          if (n >= N) break;
          T v = alpha * (h ? acc1[n] : acc0[n]);
          if (it.Cin) v += beta * cin[u];
          it.C[row + (long long)n * it.ldc] = v;
        }
      }
    }
  }
}

// ---------------------------------------------------------------- TN
template <typename T>
__global__ void __launch_bounds__(kTNThreads)
    skinny_tn2_kernel(const GemmItem<T, T> *__restrict__ items, const GemmSeg<T> *__restrict__ segs,
                      T alpha, T beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tn2_unit<T>(items, segs, alpha, beta, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// ---------------------------------------------------------------- FP64 on the DMMA pipe
// FP64 items of at most 16 columns (the HODLR matvec's D x + U t and V^T x)
// run on the FP64 tensor-core instruction mma.m16n8k4.f64: one instruction
// per 16 x 8 x 4 block instead of 512 FMAs, so the kernels stay bound by the
// operand stream instead of by instruction issue.  Fragments (PTX layout of
// m16n8k4 .f64, g = lane / 4, t = lane % 4): A a0 = A[g][t], a1 = A[g + 8][t];
// B b = B[t][g]; C c0..c3 = C[g][2t], C[g][2t + 1], C[g + 8][2t], C[g + 8][2t + 1].
__device__ inline void dmma(double (&c)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
      "{%0, %1, %2, %3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b));
}

constexpr int kDmmaRows = 512;          // NN: 8 warps x 64 rows
constexpr int kDmmaKT = 8;              // NN: K per stage
constexpr int kDmmaStages = 3;
constexpr int kDmmaAP = kDmmaRows + 8;  // padded k-row stride (doubles)

// NN: C (M x N) = beta Cin + alpha sum_s A_s B_s, A_s column-major; one CTA
// per (item, 512-row block, block of 8 NT8 columns)
template <int NT8>
__global__ void __launch_bounds__(kSkThreads, 2)
    skinny_nn_dmma_kernel(const GemmItem<double, double> *__restrict__ items,
                          const GemmSeg<double> *__restrict__ segs, double alpha, double beta) {
  constexpr int KT = kDmmaKT, ROWS = kDmmaRows, AP = kDmmaAP, NCS = 8 * NT8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);      // [stage][KT][AP]
  double *Bs = As + (size_t)kDmmaStages * KT * AP;         // [stage][KT][NCS]
  const GemmItem<double, double> it = items[blockIdx.x];
  const int row0 = blockIdx.y * ROWS;
  const int n0 = blockIdx.z * NCS;  // column block of this CTA
  if (row0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int N = it.N - n0;  // columns left from n0

  auto load = [&](const TileIter<double> &p, int st) {
    if (p.valid) {
      const GemmSeg<double> &sg = p.sg;
      double *a = As + (size_t)st * KT * AP;
      double *b = Bs + (size_t)st * KT * NCS;
      const double *abase = sg.A + row0 + (long long)p.k0 * sg.lda;
      const bool vec = ((reinterpret_cast<uintptr_t>(abase) & 15) == 0) && ((sg.lda & 1) == 0);
      for (int e = tid; e < KT * (ROWS / 2); e += kSkThreads) {
        const int k = e / (ROWS / 2), rv = e % (ROWS / 2);
        const int r = row0 + 2 * rv;
        const bool kin = p.k0 + k < sg.K;
        const double *src = abase + 2 * rv + (long long)k * sg.lda;
        double *dst = a + k * AP + 2 * rv;
        if (vec && kin && r + 2 <= it.M) {
          cpa(dst, src, 16, true);
        } else {
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const bool ok = kin && r + u < it.M;
            cpa(dst + u, ok ? src + u : sg.A, 8, ok);
          }
        }
      }
      for (int e = tid; e < KT * NCS; e += kSkThreads) {
        const int k = e % KT, n = e / KT;
        const bool ok = (p.k0 + k < sg.K) && n < N;
        cpa(b + k * NCS + n, ok ? sg.B + (p.k0 + k) + (long long)(n0 + n) * sg.ldb : sg.B, 8,
            ok);
      }
    }
    cpa_commit();
  };

  double acc[4][NT8][4];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT8; ++nt)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[mt][nt][v] = 0.0;
  TileIter<double> ld, cp;
  ld.init(segs, it.seg_begin, it.seg_count);
  cp = ld;
#pragma unroll
  for (int i = 0; i < kDmmaStages - 1; ++i) {
    load(ld, i);
    if (ld.valid) ld.next(KT);
  }
  int st = 0, lst = kDmmaStages - 1;
  const int wrow = warp * 64;
  while (cp.valid) {
    load(ld, lst);
    if (ld.valid) ld.next(KT);
    lst = (lst + 1) % kDmmaStages;
    cpa_wait<kDmmaStages - 1>();
    __syncthreads();
    const double *a = As + (size_t)st * KT * AP;
    const double *b = Bs + (size_t)st * KT * NCS;
#pragma unroll
    for (int ks = 0; ks < KT; ks += 4) {
      const double *ak = a + (ks + t) * AP + wrow + g;
      double bv[NT8];
#pragma unroll
      for (int nt = 0; nt < NT8; ++nt) bv[nt] = b[(ks + t) * NCS + nt * 8 + g];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const double a0 = ak[mt * 16], a1 = ak[mt * 16 + 8];
#pragma unroll
        for (int nt = 0; nt < NT8; ++nt) dmma(acc[mt][nt], a0, a1, bv[nt]);
      }
    }
    __syncthreads();  // stage st is refilled kDmmaStages - 1 tiles later
    st = (st + 1) % kDmmaStages;
    cp.next(KT);
  }
  cpa_wait<0>();
  // per 16-row fragment: its Cin values before its stores (C may alias Cin,
  // so a load after a store would wait for it)
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    double cin[NT8][4];
#pragma unroll
    for (int nt = 0; nt < NT8; ++nt)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = row0 + wrow + mt * 16 + g + (v >> 1) * 8;
        const int c = nt * 8 + 2 * t + (v & 1);
        cin[nt][v] = (it.Cin && row < it.M && c < N) ? it.Cin[row + (n0 + c) * (long long)it.ldcin]
                                                      : 0.0;
      }
#pragma unroll
    for (int nt = 0; nt < NT8; ++nt)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = row0 + wrow + mt * 16 + g + (v >> 1) * 8;
        const int c = nt * 8 + 2 * t + (v & 1);
        if (row < it.M && c < N) {
          const long long col = n0 + c;
          double val = alpha * acc[mt][nt][v];
          if (it.Cin) val += beta * cin[nt][v];
          it.C[row + col * it.ldc] = val;
        }
      }
  }
}

// TN: C (64 x 16 block of an item, over all K) = beta Cin + alpha sum_s A_s^T B_s
constexpr int kDmmaKC = 32;
constexpr int kDmmaLDK = kDmmaKC + 4;  // padded k stride (doubles): conflict-free fragments

__global__ void __launch_bounds__(kTNThreads)
    skinny_tn_dmma_kernel(const GemmItem<double, double> *__restrict__ items,
                          const GemmSeg<double> *__restrict__ segs, double alpha, double beta) {
  constexpr int TM = 64, TN = 16, KC = kDmmaKC, LDK = kDmmaLDK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);   // [stage][TM][LDK]
  double *Bs = As + (size_t)kSkStages * TM * LDK;      // [stage][TN][LDK]
  const GemmItem<double, double> it = items[blockIdx.x];
  const int m0 = blockIdx.y * TM, n0 = blockIdx.z * TN;
  if (m0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;

  auto load_block = [&](double *dst, const double *base, long long ld, int k0, int K, int c0,
                        int ncols, int cmax) {
    const double *p0 = base + k0 + (long long)c0 * ld;
    const bool vec = ((reinterpret_cast<uintptr_t>(p0) & 15) == 0) && ((ld & 1) == 0);
    for (int e = tid; e < ncols * (KC / 2); e += kTNThreads) {
      const int c = e / (KC / 2), kv = e % (KC / 2);
      const int k = k0 + 2 * kv;
      const bool colok = c0 + c < cmax;
      const double *src = p0 + 2 * kv + (long long)c * ld;
      double *d = dst + c * LDK + 2 * kv;
      if (vec && colok && k + 2 <= K) {
        cpa(d, src, 16, true);
      } else {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const bool ok = colok && k + u < K;
          cpa(d + u, ok ? src + u : base, 8, ok);
        }
      }
    }
  };
  auto load = [&](const TileIter<double> &p, int st) {
    if (p.valid) {
      load_block(As + (size_t)st * TM * LDK, p.sg.A, p.sg.lda, p.k0, p.sg.K, m0, TM, it.M);
      load_block(Bs + (size_t)st * TN * LDK, p.sg.B, p.sg.ldb, p.k0, p.sg.K, n0, TN, it.N);
    }
    cpa_commit();
  };

  double acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
  TileIter<double> ld, cp;
  ld.init(segs, it.seg_begin, it.seg_count);
  cp = ld;
#pragma unroll
  for (int i = 0; i < kSkStages - 1; ++i) {
    load(ld, i);
    if (ld.valid) ld.next(KC);
  }
  int st = 0, lst = kSkStages - 1;
  while (cp.valid) {
    load(ld, lst);
    if (ld.valid) ld.next(KC);
    lst = (lst + 1) % kSkStages;
    cpa_wait<kSkStages - 1>();
    __syncthreads();
    const double *a = As + (size_t)st * TM * LDK + (warp * 16 + g) * LDK + t;
    const double *b = Bs + (size_t)st * TN * LDK + g * LDK + t;
#pragma unroll
    for (int ks = 0; ks < KC; ks += 4) {
      const double a0 = a[ks], a1 = a[8 * LDK + ks];
      dmma(acc[0], a0, a1, b[ks]);
      dmma(acc[1], a0, a1, b[8 * LDK + ks]);
    }
    __syncthreads();
    st = (st + 1) % kSkStages;
    cp.next(KC);
  }
  cpa_wait<0>();
  // every Cin value before any store (C may alias Cin)
  double cin[2][4];
#pragma unroll
  for (int nt = 0; nt < 2; ++nt)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int gm = m0 + warp * 16 + g + (v >> 1) * 8;
      const int gn = n0 + nt * 8 + 2 * t + (v & 1);
      cin[nt][v] = (it.Cin && gm < it.M && gn < it.N) ? it.Cin[gm + (long long)gn * it.ldcin] : 0.0;
    }
#pragma unroll
  for (int nt = 0; nt < 2; ++nt)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int gm = m0 + warp * 16 + g + (v >> 1) * 8;
      const int gn = n0 + nt * 8 + 2 * t + (v & 1);
      if (gm < it.M && gn < it.N) {
        double val = alpha * acc[nt][v];
        if (it.Cin) val += beta * cin[nt][v];
        it.C[gm + (long long)gn * it.ldc] = val;
      }
    }
}

}  // namespace

template <typename T>
void launch_skinny(const GemmItem<T, T> *items, const GemmSeg<T> *segs, int nitems, int max_m,
                   int max_n, bool trans, T alpha, T beta, cudaStream_t s) {
  if (nitems <= 0 || max_m <= 0 || max_n <= 0) return;
  if constexpr (sizeof(T) == 8) {
    // FP64 products run on the FP64 tensor pipe (DMMA)
    if (trans) {
      const size_t smem = (size_t)kSkStages * (64 + 16) * kDmmaLDK * sizeof(double);
      raise_smem_limit(reinterpret_cast<const void *>(skinny_tn_dmma_kernel), smem);
      dim3 grid(nitems, cdiv(max_m, 64), cdiv(max_n, 16));
      skinny_tn_dmma_kernel<<<grid, kTNThreads, smem, s>>>(items, segs, alpha, beta);
    } else {
      // 8 columns per CTA when every item has at most 8, else 16-column blocks
      dim3 grid(nitems, cdiv(max_m, kDmmaRows), max_n <= 8 ? 1 : cdiv(max_n, 16));
      auto go = [&](auto kern, int ncs) {
        const size_t smem = (size_t)kDmmaStages * kDmmaKT * (kDmmaAP + ncs) * sizeof(double);
        raise_smem_limit(reinterpret_cast<const void *>(kern), smem);
        kern<<<grid, kSkThreads, smem, s>>>(items, segs, alpha, beta);
      };
      if (max_n <= 8) go(skinny_nn_dmma_kernel<1>, 8);
      else go(skinny_nn_dmma_kernel<2>, 16);
    }
    HODLR_LAUNCH_CHECK();
    return;
  }
  if (trans) {
    constexpr int TM = 64, TN = 16;
    const size_t smem = tn2_smem_bytes<T>();
    raise_smem_limit(reinterpret_cast<const void *>(skinny_tn2_kernel<T>), smem);
    dim3 grid(nitems, cdiv(max_m, TM), cdiv(max_n, TN));
    skinny_tn2_kernel<T><<<grid, kTNThreads, smem, s>>>(items, segs, alpha, beta);
  } else if constexpr (sizeof(T) == 4) {
    const int rbn = cdiv(max_m, kRowThreads);
    const long long nunits = (long long)nitems * rbn;
    if (nunits > 0x7fffffffLL) throw CudaError{cudaErrorInvalidValue};
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    const int grid = (int)std::min<long long>(nunits, 3LL * sms);
    const int nu = (int)nunits;
    const auto *fi = reinterpret_cast<const GemmItem<float, float> *>(items);
    const auto *fs = reinterpret_cast<const GemmSeg<float> *>(segs);
    if (max_n <= 8)
      skinny_nn_rows_kernel<8><<<grid, kRowThreads, 0, s>>>(fi, fs, alpha, beta, nu, rbn);
    else if (max_n <= 16)
      skinny_nn_rows_kernel<16><<<grid, kRowThreads, 0, s>>>(fi, fs, alpha, beta, nu, rbn);
    else
      skinny_nn_rows_kernel<32><<<grid, kRowThreads, 0, s>>>(fi, fs, alpha, beta, nu, rbn);
  } else {
    constexpr int KT = nn_kt<T>();
    dim3 grid(nitems, cdiv(max_m, kNNRows));
    if (max_n <= 16) {
      const size_t smem = (size_t)nn_stages<T>() * KT * (kNNRows + 16) * sizeof(T);
      raise_smem_limit(reinterpret_cast<const void *>(skinny_nn2_kernel<T, 16>), smem);
      skinny_nn2_kernel<T, 16><<<grid, kSkThreads, smem, s>>>(items, segs, alpha, beta);
    } else {
      const size_t smem = (size_t)nn_stages<T>() * KT * (kNNRows + 32) * sizeof(T);
      raise_smem_limit(reinterpret_cast<const void *>(skinny_nn2_kernel<T, 32>), smem);
      skinny_nn2_kernel<T, 32><<<grid, kSkThreads, smem, s>>>(items, segs, alpha, beta);
    }
  }
  HODLR_LAUNCH_CHECK();
}

template void launch_skinny<double>(const GemmItem<double, double> *, const GemmSeg<double> *,
                                    int, int, int, bool, double, double, cudaStream_t);
template void launch_skinny<float>(const GemmItem<float, float> *, const GemmSeg<float> *, int,
                                   int, int, bool, float, float, cudaStream_t);

}  // namespace hodlr
