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
#include "common.cuh"
#include "gemm_skinny.cuh"

namespace hodlr {

namespace {

constexpr int kSkThreads = 256;
constexpr int kSkStages = 3;

__device__ inline void cpa(void *dst, const void *src, int bytes, bool ok) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = ok ? bytes : 0;
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n));
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n));
}
__device__ inline void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The K tiles of an item, flattened over its segments (zero-length ones skipped).
template <typename T>
struct TileIter {
  const GemmSeg<T> *segs;
  int s, s_end, k0;
  GemmSeg<T> sg;
  bool valid;
  __device__ void init(const GemmSeg<T> *sp, int b, int c) {
    segs = sp;
    s = b;
    s_end = b + c;
    k0 = 0;
    settle();
  }
  __device__ void settle() {
    valid = false;
    for (; s < s_end; ++s) {
      sg = segs[s];
      if (sg.K > 0) { valid = true; return; }
    }
  }
  __device__ void next(int kt) {
    k0 += kt;
    if (k0 < sg.K) return;
    k0 = 0;
    ++s;
    settle();
  }
};

template <typename T>
struct Vec {
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  static constexpr int W = 16 / sizeof(T);
};

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
#pragma unroll
      for (int n = 0; n < NC; ++n) {
        if (n >= N) break;
        T v = alpha * (h ? acc1[n] : acc0[n]);
        if (it.Cin) v += beta * it.Cin[row + (long long)n * it.ldcin];
        it.C[row + (long long)n * it.ldc] = v;
      }
    }
  }
}

// ---------------------------------------------------------------- TN
constexpr int kTNThreads = 128;

template <typename T>
__global__ void __launch_bounds__(kTNThreads)
    skinny_tn2_kernel(const GemmItem<T, T> *__restrict__ items, const GemmSeg<T> *__restrict__ segs,
                      T alpha, T beta) {
  constexpr int TM = 64, TN = 16, KC = 32;
  constexpr int VW = Vec<T>::W;
  constexpr int LDK = KC + VW;  // padded k stride (16-byte multiple)
  using V = typename Vec<T>::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *As = reinterpret_cast<T *>(smem_raw);          // [stage][TM][LDK]
  T *Bs = As + (size_t)kSkStages * TM * LDK;        // [stage][TN][LDK]
  const GemmItem<T, T> it = items[blockIdx.x];
  const int m0 = blockIdx.y * TM, n0 = blockIdx.z * TN;
  if (m0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x;
  const int mm = tid & 31, n4 = (tid >> 5) * 4;  // rows mm, mm + 32; columns n4 .. n4 + 3

  // rows (k) of a K x cols operand block, k-contiguous, into dst[col][LDK]
  auto load_block = [&](T *dst, const T *base, long long ld, int k0, int K, int c0, int ncols,
                        int cmax) {
    const T *p0 = base + k0 + (long long)c0 * ld;
    const bool vec = ((reinterpret_cast<uintptr_t>(p0) & 15) == 0) && ((ld % VW) == 0);
    if (vec) {
      for (int e = tid; e < ncols * (KC / VW); e += kTNThreads) {
        const int c = e / (KC / VW), kv = e % (KC / VW);
        const int k = k0 + kv * VW;
        const bool colok = c0 + c < cmax;
        const T *src = p0 + kv * VW + (long long)c * ld;
        if (colok && k + VW <= K) {
          cpa(dst + c * LDK + kv * VW, src, 16, true);
        } else {
#pragma unroll
          for (int u = 0; u < VW; ++u) {
            const bool ok = colok && k + u < K;
            cpa(dst + c * LDK + kv * VW + u, ok ? src + u : base, sizeof(T), ok);
          }
        }
      }
    } else {
      for (int e = tid; e < ncols * KC; e += kTNThreads) {
        const int c = e / KC, kk = e % KC;
        const bool ok = c0 + c < cmax && k0 + kk < K;
        cpa(dst + c * LDK + kk, ok ? p0 + kk + (long long)c * ld : base, sizeof(T), ok);
      }
    }
  };
  auto load = [&](const TileIter<T> &p, int st) {
    if (p.valid) {
      load_block(As + (size_t)st * TM * LDK, p.sg.A, p.sg.lda, p.k0, p.sg.K, m0, TM, it.M);
      load_block(Bs + (size_t)st * TN * LDK, p.sg.B, p.sg.ldb, p.k0, p.sg.K, n0, TN, it.N);
    }
    cpa_commit();
  };

  T acc[2][4] = {{T(0), T(0), T(0), T(0)}, {T(0), T(0), T(0), T(0)}};
  TileIter<T> ld, cp;
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
    const T *a = As + (size_t)st * TM * LDK + mm * LDK;
    const T *b = Bs + (size_t)st * TN * LDK + n4 * LDK;
#pragma unroll
    for (int kv = 0; kv < KC / VW; ++kv) {
      const V av0 = *reinterpret_cast<const V *>(a + kv * VW);
      const V av1 = *reinterpret_cast<const V *>(a + 32 * LDK + kv * VW);
      const T *ap0 = reinterpret_cast<const T *>(&av0);
      const T *ap1 = reinterpret_cast<const T *>(&av1);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const V bv = *reinterpret_cast<const V *>(b + j * LDK + kv * VW);
        const T *bp = reinterpret_cast<const T *>(&bv);
#pragma unroll
        for (int u = 0; u < VW; ++u) {
          acc[0][j] += ap0[u] * bp[u];
          acc[1][j] += ap1[u] * bp[u];
        }
      }
    }
    __syncthreads();
    st = (st + 1) % kSkStages;
    cp.next(KC);
  }
  cpa_wait<0>();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int gm = m0 + mm + 32 * h;
    if (gm >= it.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + n4 + j;
      if (gn >= it.N) break;
      T v = alpha * acc[h][j];
      if (it.Cin) v += beta * it.Cin[gm + (long long)gn * it.ldcin];
      it.C[gm + (long long)gn * it.ldc] = v;
    }
  }
}

}  // namespace

template <typename T>
void launch_skinny(const GemmItem<T, T> *items, const GemmSeg<T> *segs, int nitems, int max_m,
                   int max_n, bool trans, T alpha, T beta, cudaStream_t s) {
  if (nitems <= 0 || max_m <= 0 || max_n <= 0) return;
  if (trans) {
    constexpr int TM = 64, TN = 16, KC = 32, LDK = KC + 16 / sizeof(T);
    const size_t smem = (size_t)kSkStages * (TM + TN) * LDK * sizeof(T);
    HODLR_CUDA_TRY(cudaFuncSetAttribute(skinny_tn2_kernel<T>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid(nitems, cdiv(max_m, TM), cdiv(max_n, TN));
    skinny_tn2_kernel<T><<<grid, kTNThreads, smem, s>>>(items, segs, alpha, beta);
  } else {
    constexpr int KT = nn_kt<T>();
    dim3 grid(nitems, cdiv(max_m, kNNRows));
    if (max_n <= 16) {
      const size_t smem = (size_t)nn_stages<T>() * KT * (kNNRows + 16) * sizeof(T);
      HODLR_CUDA_TRY(cudaFuncSetAttribute(skinny_nn2_kernel<T, 16>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      skinny_nn2_kernel<T, 16><<<grid, kSkThreads, smem, s>>>(items, segs, alpha, beta);
    } else {
      const size_t smem = (size_t)nn_stages<T>() * KT * (kNNRows + 32) * sizeof(T);
      HODLR_CUDA_TRY(cudaFuncSetAttribute(skinny_nn2_kernel<T, 32>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
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
