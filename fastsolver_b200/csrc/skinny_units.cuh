// skinny_units.cuh -- CTA-level building blocks of the skinny GEMM items
// (at most 32 columns: the refinement sweeps' reduce, node apply and
// broadcast), shared by the one-launch-per-step kernels of gemm_skinny.cu and
// the persistent level-walk kernel of sweep.cu.  Every unit is executed by all
// threads of a CTA together (it synchronizes the CTA) and returns early only
// CTA-uniformly.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace hodlr {
namespace sk {

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

// Global loads of the units.  CG = false: the read-only path (__ldg), for
// one-step kernels whose inputs are never written by the same launch.
// CG = true: L2-only loads (__ldcg), for the persistent level-walk kernel,
// whose later steps read what other CTAs wrote in earlier steps of the same
// launch (an L1 or read-only-cache copy of an earlier step's value would be
// stale).
template <bool CG, typename T>
__device__ inline T ldg_unit(const T *p) {
  if constexpr (CG) return __ldcg(p);
  else return __ldg(p);
}

template <typename T>
struct Vec {
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  static constexpr int W = 16 / sizeof(T);
};

// ---------------------------------------------------------------- NN (rows)
// FP32 C (M x N <= NC) = beta Cin + alpha sum_s A_s B_s with one row per
// thread: A is read straight from global memory (a warp reads 32 consecutive
// rows of one column: 128 bytes), 32 (16 when NC = 32) k-values in flight
// per thread, while the matching block of B sits in shared memory.  Small CTAs (128 rows)
// and no A staging let many CTAs share an SM, which keeps enough loads in
// flight for the short-K products of the refinement sweeps (K = r).
constexpr int kRowThreads = 128;

template <int NC>
// k-values in flight per thread (a whole K = 64 chunk for up to 16 columns
// made the persistent sweep spill and run slower: 2.02 -> 2.12 ms for two
// sweeps at N = 262144)
__host__ __device__ constexpr int nn_rows_kc() { return NC > 16 ? 16 : 32; }

// One CTA (kRowThreads threads) computes rows [rb * kRowThreads, ...) of item
// `item`; Bs holds nn_rows_kc<NC>() * NC floats.  CTA-uniform.
template <int NC, bool CG = false>
__device__ inline void nn_rows_unit(const GemmItem<float, float> *__restrict__ items,
                                    const GemmSeg<float> *__restrict__ segs, float alpha,
                                    float beta, int item, int rb, float *Bs) {
  constexpr int kRowKC = nn_rows_kc<NC>();
  const GemmItem<float, float> it = items[item];
  const int row0 = rb * kRowThreads;
  if (row0 >= it.M) return;
  const int tid = threadIdx.x;
  const int row = row0 + tid;
  const bool live = row < it.M;
  const int N = it.N;
  float acc[NC];
#pragma unroll
  for (int n = 0; n < NC; ++n) acc[n] = 0.f;
  for (int sidx = it.seg_begin; sidx < it.seg_begin + it.seg_count; ++sidx) {
    const GemmSeg<float> sg = segs[sidx];
    for (int k0 = 0; k0 < sg.K; k0 += kRowKC) {
      const int kc = min(kRowKC, sg.K - k0);
      // this chunk's A values of the thread's row (issued before the barrier)
      float a[kRowKC];
      const float *ap = sg.A + (live ? row : 0) + (long long)k0 * sg.lda;
#pragma unroll
      for (int k = 0; k < kRowKC; ++k)
        a[k] = (k < kc) ? ldg_unit<CG>(ap + (long long)k * sg.lda) : 0.f;
      // ... and this thread's share of the chunk's B block, in flight with them
      constexpr int kBPer = kRowKC * NC / kRowThreads;
      static_assert(kBPer * kRowThreads == kRowKC * NC, "whole B block per pass");
      float bv[kBPer];
#pragma unroll
      for (int j = 0; j < kBPer; ++j) {
        const int e = tid + j * kRowThreads;
        const int k = e % kRowKC, n = e / kRowKC;
        bv[j] = (k < kc && n < N) ? ldg_unit<CG>(sg.B + (k0 + k) + (long long)n * sg.ldb) : 0.f;
      }
      __syncthreads();  // the previous chunk's B reads are done
#pragma unroll
      for (int j = 0; j < kBPer; ++j) {
        const int e = tid + j * kRowThreads;
        Bs[(e % kRowKC) * NC + e / kRowKC] = bv[j];
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kRowKC; ++k) {
#pragma unroll
        for (int n = 0; n < NC; n += 4) {
          const float4 b = *reinterpret_cast<const float4 *>(Bs + k * NC + n);
          acc[n] += a[k] * b.x;
          acc[n + 1] += a[k] * b.y;
          acc[n + 2] += a[k] * b.z;
          acc[n + 3] += a[k] * b.w;
        }
      }
    }
  }
  if (!live) return;
  // all of the row's Cin values before any store: C may be Cin (in-place
  // d -= u eta), so loads issued between the stores would each wait for the
  // one before
  float cin[NC];
  if (it.Cin) {
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const float *cp = it.Cin + row + (long long)n * it.ldcin;
      cin[n] = n < N ? (CG ? __ldcg(cp) : *cp) : 0.f;
    }
  }
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    if (n >= N) break;
    float v = alpha * acc[n];
    if (it.Cin) v += beta * cin[n];
    it.C[row + (long long)n * it.ldc] = v;
  }
}


// ---------------------------------------------------------------- TN
constexpr int kTNThreads = 128;

template <typename T>
__host__ __device__ constexpr size_t tn2_smem_bytes() {
  return (size_t)kSkStages * (64 + 16) * (32 + 16 / sizeof(T)) * sizeof(T);
}

// One CTA (kTNThreads threads) computes the 64 x 16 block (mt, nt) of item
// `item` over all of its K; smem holds tn2_smem_bytes<T>().  CTA-uniform.
template <typename T, bool CG = false>
__device__ inline void tn2_unit(const GemmItem<T, T> *__restrict__ items,
                                const GemmSeg<T> *__restrict__ segs, T alpha, T beta, int item,
                                int mt, int nt, unsigned char *smem_raw) {
  constexpr int TM = 64, TN = 16, KC = 32;
  constexpr int VW = Vec<T>::W;
  constexpr int LDK = KC + VW;  // padded k stride (16-byte multiple)
  using V = typename Vec<T>::V;
  T *As = reinterpret_cast<T *>(smem_raw);          // [stage][TM][LDK]
  T *Bs = As + (size_t)kSkStages * TM * LDK;        // [stage][TN][LDK]
  const GemmItem<T, T> it = items[item];
  const int m0 = mt * TM, n0 = nt * TN;
  if (m0 >= it.M || n0 >= it.N) return;
  const int tid = threadIdx.x;
  const int mm = tid & 31, n4 = (tid >> 5) * 4;  // rows mm, mm + 32; columns n4 .. n4 + 3

  // one element: asynchronous (L1-allocating) copy, or with CG an L2 load
  // stored directly (it is read after the same cp.async wait and barrier)
  auto elem = [&](T *dst, const T *src, bool ok) {
    if constexpr (CG) *dst = ok ? __ldcg(src) : T(0);
    else cpa(dst, src, sizeof(T), ok);
  };
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
            elem(dst + c * LDK + kv * VW + u, ok ? src + u : base, ok);
          }
        }
      }
    } else {
      for (int e = tid; e < ncols * KC; e += kTNThreads) {
        const int c = e / KC, kk = e % KC;
        const bool ok = c0 + c < cmax && k0 + kk < K;
        elem(dst + c * LDK + kk, ok ? p0 + kk + (long long)c * ld : base, ok);
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
  // every Cin value before any store (C may be Cin)
  T cin[2][4];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gm = m0 + mm + 32 * h, gn = n0 + n4 + j;
      const T *cp = it.Cin ? it.Cin + gm + (long long)gn * it.ldcin : nullptr;
      cin[h][j] = (cp && gm < it.M && gn < it.N) ? (CG ? __ldcg(cp) : *cp) : T(0);
    }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int gm = m0 + mm + 32 * h;
    if (gm >= it.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + n4 + j;
      if (gn >= it.N) break;
      T v = alpha * acc[h][j];
      if (it.Cin) v += beta * cin[h][j];
      it.C[gm + (long long)gn * it.ldc] = v;
    }
  }
}

}  // namespace sk
}  // namespace hodlr
