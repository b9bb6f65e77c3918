// leaf_blocked.cu -- batched blocked leaf factorization on [D | X].
//
// The leaf task body (src/solver/solver_tasks.cc:424-450) is dgesv(D, X) on
// all m + r*L columns of the leaf.  On the GPU every leaf of the tree is
// factored at once, panel by panel (NB columns), as a right-looking blocked
// LU of the augmented matrix [D | X]:
//
//   for each panel k0:
//     leaf_panel_kernel   one CTA per leaf: LU with partial pivoting of
//                         D[k0:n, k0:k0+NB] in shared memory (LAPACK idamax
//                         tie rule), written back; the inverses of the
//                         panel's unit-lower and upper diagonal blocks are
//                         formed (one thread per column) for the solves;
//                         ipiv / perm updated, per-leaf "had interchanges" flag
//     leaf_laswp_kernel   the panel's row interchanges on every other column
//                         of D (LAPACK layout) and of X; a no-op for leaves
//                         whose panel pivoted on the diagonal
//     batched GEMM        U12 = L11^{-1} A12 (in place, D and X columns)
//     batched GEMM        A22 -= L21 U12 (D trailing block and X rows below)
//   then for each panel from the last: X[k] = U_kk^{-1} X[k];
//                                      X[0:k0] -= U[0:k0, k] X[k]
// so D ends as LAPACK's P L U factors, X as D^{-1} X.  The GEMMs are items of
// the batched GEMM engine (gemm_simt.cu), one launch per step for all leaves.
#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "leaf_blocked.cuh"

namespace hodlr {

namespace {

constexpr int kThreads = 256;

// 16-byte vector of T
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using V = float4;
};
template <>
struct Vec16<double> {
  using V = double2;
};

template <typename T>
__device__ inline T tabs(T v) {
  return v < T(0) ? -v : v;
}

// Panel LU with implicit row interchanges.  Thread t owns the panel rows
// t, t + 256, ... (storage order, never moved in shared memory) and tracks
// each row's position in LAPACK's current row order.  Column j: every warp
// finds its best candidate (largest |a|, lowest current position on ties,
// as idamax), one barrier, every thread combines the 8 warp results, reads
// the pivot row and eliminates its own rows; the row at position j takes the
// pivot's old position (the interchange) and the pivot takes position j.
// One barrier per column.  At the end the rows are written to D in their
// final order, which is exactly dgetf2's.
template <typename T, int NB>
__global__ void __launch_bounds__(kThreads)
    leaf_panel_kernel(const LeafFactorTask<T> *__restrict__ tasks, int k0, int panel,
                      int panel_stride, int *info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int RPT = 4;  // rows per thread (panel rows <= 1024)
  const LeafFactorTask<T> tk = tasks[blockIdx.x];
  const int n = tk.n;
  if (k0 >= n) return;
  const int kb = min(NB, n - k0);
  const int R = n - k0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int PS = panel_stride;
  T *P = reinterpret_cast<T *>(smem_raw);        // PS x NB, column-major, storage order
  T *Lr = P + (size_t)PS * NB;                   // NB x NB row-major
  T *Ur = Lr + NB * NB;                          // NB x NB row-major
  int *pv = reinterpret_cast<int *>(Ur + NB * NB);   // NB: pivot position per column
  int *ps = pv + NB;                                 // NB: pivot storage row per column
  T *wv = reinterpret_cast<T *>(ps + NB);            // 2 x 8 warp best values
  int *wp = reinterpret_cast<int *>(wv + 16);        // 2 x 8 warp best positions
  int *wsr = wp + 16;                                // 2 x 8 warp best storage rows
  int *dst = wsr + 16;                               // PS: final position of each row
  T *D = tk.D;
  const long long ldd = tk.ldd;
  for (int j = 0; j < kb; ++j) {
    const T *src = D + (long long)(k0 + j) * ldd + k0;
    for (int i = tid; i < R; i += kThreads) P[i + (size_t)j * PS] = src[i];
  }
  int pos[RPT];
#pragma unroll
  for (int q = 0; q < RPT; ++q) pos[q] = tid + q * kThreads;  // current positions
  auto warp_best = [&](int j, int slot) {
    T best = T(-1);
    int bp = 1 << 30, bs = -1;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int i = tid + q * kThreads;
      if (i < R && pos[q] >= j) {
        const T a = tabs(P[i + (size_t)j * PS]);
        if (a > best || (a == best && pos[q] < bp)) { best = a; bp = pos[q]; bs = i; }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const T ob = __shfl_down_sync(0xffffffffu, best, off);
      const int op = __shfl_down_sync(0xffffffffu, bp, off);
      const int os = __shfl_down_sync(0xffffffffu, bs, off);
      if (ob > best || (ob == best && op < bp)) { best = ob; bp = op; bs = os; }
    }
    if (lane == 0) { wv[slot * 8 + warp] = best; wp[slot * 8 + warp] = bp; wsr[slot * 8 + warp] = bs; }
  };
  __syncthreads();
  warp_best(0, 0);
  __syncthreads();
  int info_local = 0;
  bool swaps = false;
  for (int j = 0; j < kb; ++j) {
    const int slot = j & 1;
    // combine the warp candidates (every thread, same result)
    T b = wv[slot * 8];
    int p = wp[slot * 8], sp = wsr[slot * 8];
#pragma unroll
    for (int w = 1; w < kThreads / 32; ++w) {
      const T v = wv[slot * 8 + w];
      const int vp = wp[slot * 8 + w];
      if (v > b || (v == b && vp < p)) { b = v; p = vp; sp = wsr[slot * 8 + w]; }
    }
    if (sp < 0) { p = j; sp = -1; }  // no candidate (all NaN): keep position j
    if (tid == 0) { pv[j] = p; ps[j] = sp; }
    if (p != j) swaps = true;
    // interchange: the row at position j moves to p, the pivot row to j
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int i = tid + q * kThreads;
      if (i < R) {
        if (pos[q] == j && i != sp) pos[q] = p;
        else if (i == sp) pos[q] = j;
      }
    }
    const T piv = sp >= 0 ? P[sp + (size_t)j * PS] : T(0);
    if (piv == T(0)) {
      if (info_local == 0) info_local = k0 + j + 1;
    } else {
      const T rinv = T(1) / piv;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int i = tid + q * kThreads;
        if (i < R && pos[q] > j) {
          const T l = P[i + (size_t)j * PS] * rinv;
          P[i + (size_t)j * PS] = l;
          for (int c = j + 1; c < kb; ++c) P[i + (size_t)c * PS] -= l * P[sp + (size_t)c * PS];
        }
      }
    }
    if (j + 1 < kb) warp_best(j + 1, slot ^ 1);
    __syncthreads();
  }
  // write the rows back in their final order; build the diagonal block
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int i = tid + q * kThreads;
    if (i < R) dst[i] = pos[q];
  }
  __syncthreads();
  for (int j = 0; j < kb; ++j) {
    T *col = D + (long long)(k0 + j) * ldd + k0;
    for (int i = tid; i < R; i += kThreads) col[dst[i]] = P[i + (size_t)j * PS];
  }
  for (int e = tid; e < NB * NB; e += kThreads) { Lr[e] = T(0); Ur[e] = T(0); }
  __syncthreads();
  for (int i = tid; i < R; i += kThreads) {
    const int r = dst[i];
    if (r < kb)
      for (int k = 0; k < kb; ++k) {
        const T v = P[i + (size_t)k * PS];
        if (k < r) Lr[r * NB + k] = v;
        else Ur[r * NB + k] = v;
      }
  }
  __syncthreads();
  for (int i = tid; i < NB; i += kThreads) {
    Lr[i * NB + i] = T(1);
    if (i >= kb) Ur[i * NB + i] = T(1);
  }
  __syncthreads();
  // inverses, one thread per column j (row-major storage: conflict-free reads)
  T *Li = Lr, *Ui = Ur;
  T *Lw = P, *Uw = P + NB * NB;  // the panel buffer is free now
  if (tid < NB) {
    const int j = tid;
    for (int i = 0; i < NB; ++i) Lw[i * NB + j] = (i == j) ? T(1) : T(0);
    for (int i = j + 1; i < NB; ++i) {
      T acc = T(0);
      for (int k = j; k < i; ++k) acc += Li[i * NB + k] * Lw[k * NB + j];
      Lw[i * NB + j] = -acc;
    }
    for (int i = 0; i < NB; ++i) Uw[i * NB + j] = T(0);
    for (int i = j; i >= 0; --i) {
      T acc = (i == j) ? T(1) : T(0);
      for (int k = i + 1; k <= j; ++k) acc -= Ui[i * NB + k] * Uw[k * NB + j];
      Uw[i * NB + j] = acc / Ui[i * NB + i];
    }
  }
  __syncthreads();
  T *Lout = tk.Linv + (size_t)panel * NB * NB;
  T *Uout = tk.Uinv + (size_t)panel * NB * NB;
  for (int e = tid; e < NB * NB; e += kThreads) {
    const int i = e % NB, k = e / NB;
    Lout[e] = Lw[i * NB + k];
    Uout[e] = Uw[i * NB + k];
  }
  if (tid == 0) {
    tk.swapflag[panel] = swaps ? 1 : 0;
    for (int j = 0; j < kb; ++j) {
      const int p = pv[j];
      tk.ipiv[k0 + j] = k0 + p + 1;
      if (p != j) {
        const int t = tk.perm[k0 + j];
        tk.perm[k0 + j] = tk.perm[k0 + p];
        tk.perm[k0 + p] = t;
      }
    }
    if (info_local && info && info[tk.info_slot] == 0) info[tk.info_slot] = info_local;
  }
}

// Register-resident panel LU, same semantics as leaf_panel_kernel (LAPACK
// dgetf2 pivot order, implicit interchanges, inverses of the diagonal block).
// 512 threads; thread t owns panel rows t + 512 q (q < RPT) in registers, so
// an elimination step touches no shared memory except the pivot row.  Per
// column: every warp finds its best candidate (largest |a|, lowest current
// position on ties) and the winning lane publishes its whole row; one
// barrier; every warp combines the candidates with four shuffles, reads the
// pivot row (broadcast) and eliminates its rows.  The loop over the NB
// columns is unrolled so that the row lives in registers.
constexpr int kRegThreads = 512;

// Warp-wide argmax of |a| with the lowest position on ties (idamax order),
// with warp reductions on the bit patterns (|a| >= 0 orders like its bits).
// In: per lane (best = |a| or anything when pos == INT_MAX, pos, code).
// Out: every lane holds the winner's (best, pos, code) and its lane index;
// pos == INT_MAX when no lane had a candidate.
__device__ inline void warp_argmax(float &best, int &pos, int &code, int &wlane) {
  const bool cand = pos != 0x7fffffff;
  const unsigned key = cand ? __float_as_uint(best) : 0u;
  const unsigned mx = __reduce_max_sync(0xffffffffu, key);
  const unsigned pm = __reduce_min_sync(0xffffffffu, key == mx ? (unsigned)pos : 0xffffffffu);
  const unsigned win = __ballot_sync(0xffffffffu, cand && key == mx && (unsigned)pos == pm);
  wlane = win ? __ffs(win) - 1 : 0;
  best = __uint_as_float(mx);
  pos = win ? (int)pm : 0x7fffffff;
  code = __shfl_sync(0xffffffffu, code, wlane);
  if (!win) code = -1;
}
__device__ inline void warp_argmax(double &best, int &pos, int &code, int &wlane) {
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

template <typename T, int NB, int RPT>
__global__ void __launch_bounds__(kRegThreads, 1)
    leaf_panel_reg_kernel(const LeafFactorTask<T> *__restrict__ tasks, int k0, int panel,
                          int *info) {
  constexpr int NW = kRegThreads / 32;
  constexpr int LDL = NB + 1;
  constexpr int VW = 16 / sizeof(T);
  using V = typename Vec16<T>::V;
  __shared__ __align__(16) T wrow[2][NW][NB];
  __shared__ T wval[2][NW];
  __shared__ int wpos[2][NW], wcode[2][NW];
  __shared__ T Lr[NB * LDL], Ur[NB * LDL];
  __shared__ T udr[NB];
  __shared__ int pv[NB];
  const LeafFactorTask<T> tk = tasks[blockIdx.x];
  const int n = tk.n;
  if (k0 >= n) return;
  const int kb = min(NB, n - k0);
  const int R = n - k0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // the launch gives one thread per row (RPT rows per thread) of the panel's
  // live part, at most kRegThreads: later panels run with fewer warps
  const int nthr = blockDim.x, nw = nthr >> 5;
  T *D = tk.D;
  const long long ldd = tk.ldd;
  T a[RPT][NB];
  int pos[RPT];
  bool live[RPT];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int i = tid + q * nthr;
    live[q] = i < R;
    pos[q] = i;
    const T *src = D + (k0 + i) + (long long)k0 * ldd;
#pragma unroll
    for (int c = 0; c < NB; ++c) a[q][c] = (live[q] && c < kb) ? src[(long long)c * ldd] : T(0);
  }
  bool warp_live = __any_sync(0xffffffffu, live[0]);
  int info_local = 0;
  bool swaps = false;
  // The columns are factored QW at a time by one unrolled body inside a
  // runtime loop (a quarter of the code of a fully unrolled panel, which
  // kept missing the instruction cache): before quarter h every row is
  // rotated left by h QW, so the quarter's columns sit at register positions
  // 0 .. QW - 1; positions QW .. NB - h QW - 1 hold the later quarters (they
  // are updated), the rest the finished ones (left alone).
  constexpr int QW = NB < 16 ? NB : 16;
  constexpr int NQ = NB / QW;
#pragma unroll 1
  for (int h = 0; h < NQ; ++h) {
    const int live_blocks = NQ - h;  // blocks of QW positions still being updated
#pragma unroll
    for (int jj = 0; jj < QW; ++jj) {
      const int j = h * QW + jj;  // panel column
      if (j < kb) {
        const int slot = j & 1;
        if (warp_live) {
          T best = T(0);
          int bp = 0x7fffffff, bc = -1;
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            if (live[q] && pos[q] >= j) {
              const T av = tabs(a[q][jj]);
              // NaN is never a candidate (as idamax, which skips it)
              if (av == av && (bp == 0x7fffffff || av > best || (av == best && pos[q] < bp))) {
                best = av; bp = pos[q]; bc = tid + q * nthr;
              }
            }
          }
          int wl;
          warp_argmax(best, bp, bc, wl);
          // the winning lane publishes its row (rotated like every row)
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            if (bc >= 0 && bc == tid + q * nthr) {
              V *dst = reinterpret_cast<V *>(wrow[slot][warp]);
#pragma unroll
              for (int cv = 0; cv < NB / VW; ++cv) {
                V v;
                T *vp = reinterpret_cast<T *>(&v);
#pragma unroll
                for (int u = 0; u < VW; ++u) vp[u] = a[q][cv * VW + u];
                dst[cv] = v;
              }
            }
          }
          if (lane == 0) { wval[slot][warp] = best; wpos[slot][warp] = bp; wcode[slot][warp] = bc; }
        } else if (lane == 0) {
          wval[slot][warp] = T(0); wpos[slot][warp] = 0x7fffffff; wcode[slot][warp] = -1;
        }
        __syncthreads();
        // combine the warp candidates (every thread, same result)
        T pb = T(0);
        int pp = 0x7fffffff, pc = -1, pw = 0;
        if (lane < nw) { pb = wval[slot][lane]; pp = wpos[slot][lane]; pc = wcode[slot][lane]; }
        warp_argmax(pb, pp, pc, pw);  // pw: the winning warp
        int p = j;
        T piv = T(0);
        if (pc >= 0) { p = pp; piv = wrow[slot][pw][jj]; }
        if (tid == 0) pv[j] = p;
        if (p != j) swaps = true;
        if (warp_live) {
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            if (live[q]) {
              if (tid + q * nthr == pc) pos[q] = j;
              else if (pos[q] == j) pos[q] = p;
            }
          }
          if (piv != T(0)) {
            const T rinv = sizeof(T) == 4 ? T(__frcp_rn(float(piv))) : T(__drcp_rn(double(piv)));
            const V *prow = reinterpret_cast<const V *>(wrow[slot][pw]);
#pragma unroll
            for (int q = 0; q < RPT; ++q) {
              if (live[q] && pos[q] > j) {
                const T l = a[q][jj] * rinv;
                a[q][jj] = l;
#pragma unroll
                for (int cv = (jj + 1) / VW; cv < NB / VW; ++cv) {
                  if (cv * VW >= QW && (cv * VW) / QW >= live_blocks) continue;
                  const V v = prow[cv];
                  const T *vp = reinterpret_cast<const T *>(&v);
                  if constexpr (sizeof(T) == 4) {
                    // pairs of columns through the packed FP32 FMA (each
                    // half rounded as the scalar a - l p); which columns
                    // change is known at compile time (jj is unrolled)
                    const float2 nl = make_float2(-float(l), -float(l));
#pragma unroll
                    for (int u = 0; u < VW; u += 2) {
                      const int c = cv * VW + u;
                      if (c > jj) {
                        const float2 r = __ffma2_rn(nl, make_float2(vp[u], vp[u + 1]),
                                                    make_float2(a[q][c], a[q][c + 1]));
                        a[q][c] = r.x;
                        a[q][c + 1] = r.y;
                      } else if (c + 1 > jj) {
                        a[q][c + 1] -= l * vp[u + 1];
                      }
                    }
                  } else {
#pragma unroll
                    for (int u = 0; u < VW; ++u)
                      if (cv * VW + u > jj) a[q][cv * VW + u] -= l * vp[u];
                  }
                }
              }
            }
          }
        }
        if (piv == T(0) && info_local == 0) info_local = k0 + j + 1;
      }
    }
    // rotate every row left by QW (after NQ rotations the order is restored)
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      T t[QW];
#pragma unroll
      for (int c = 0; c < QW; ++c) t[c] = a[q][c];
#pragma unroll
      for (int c = 0; c < NB - QW; ++c) a[q][c] = a[q][c + QW];
#pragma unroll
      for (int c = 0; c < QW; ++c) a[q][NB - QW + c] = t[c];
    }
  }
  // rows to their final positions; diagonal block rows to shared memory
  int pold[RPT];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    pold[q] = live[q] ? tk.perm[k0 + tid + q * nthr] : 0;
    if (live[q]) {
      T *dst = D + (k0 + pos[q]) + (long long)k0 * ldd;
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c < kb) dst[(long long)c * ldd] = a[q][c];
      if (pos[q] < kb) {
        const int r = pos[q];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
          Lr[r * LDL + c] = c < r ? a[q][c] : (c == r ? T(1) : T(0));
          Ur[r * LDL + c] = c >= r ? a[q][c] : T(0);
        }
      }
    }
  }
  for (int r = kb + tid; r < NB; r += nthr) {
    for (int c = 0; c < NB; ++c) {
      Lr[r * LDL + c] = c == r ? T(1) : T(0);
      Ur[r * LDL + c] = c == r ? T(1) : T(0);
    }
  }
  __syncthreads();  // every thread has read its perm entry and written its rows
#pragma unroll
  for (int q = 0; q < RPT; ++q)
    if (live[q]) tk.perm[k0 + pos[q]] = pold[q];
  for (int j = tid; j < kb; j += nthr) tk.ipiv[k0 + j] = k0 + pv[j] + 1;
  for (int r = tid; r < NB; r += nthr) udr[r] = T(1) / Ur[r * LDL + r];
  if (tid == 0) {
    tk.swapflag[panel] = swaps ? 1 : 0;
    if (info_local && info && info[tk.info_slot] == 0) info[tk.info_slot] = info_local;
  }
  __syncthreads();
  // inverses of the diagonal block, four columns per warp pass: lanes hold
  // rows lane + 32 r of the columns; x_k is broadcast with a shuffle
  constexpr int RPL = (NB + 31) / 32;
  T *Lout = tk.Linv + (size_t)panel * NB * NB;
  T *Uout = tk.Uinv + (size_t)panel * NB * NB;
  for (int j0 = warp * 4; j0 < NB; j0 += nw * 4) {
    T x[4][RPL];
    // L^{-1}: forward substitution on e_j
#pragma unroll
    for (int cc = 0; cc < 4; ++cc)
#pragma unroll
      for (int r = 0; r < RPL; ++r) x[cc][r] = (lane + 32 * r == j0 + cc) ? T(1) : T(0);
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      T xk[4];
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) xk[cc] = __shfl_sync(0xffffffffu, x[cc][k / 32], k % 32);
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (i > k && i < NB) {
          const T l = Lr[i * LDL + k];
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) x[cc][r] -= l * xk[cc];
        }
      }
    }
#pragma unroll
    for (int cc = 0; cc < 4; ++cc)
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (i < NB && j0 + cc < NB) Lout[i + (j0 + cc) * NB] = x[cc][r];
      }
    // U^{-1}: back substitution on e_j
#pragma unroll
    for (int cc = 0; cc < 4; ++cc)
#pragma unroll
      for (int r = 0; r < RPL; ++r) x[cc][r] = (lane + 32 * r == j0 + cc) ? T(1) : T(0);
#pragma unroll
    for (int k = NB - 1; k >= 0; --k) {
      T xk[4];
      const T dk = udr[k];
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        xk[cc] = __shfl_sync(0xffffffffu, x[cc][k / 32], k % 32) * dk;
        if (lane == k % 32) x[cc][k / 32] = xk[cc];
      }
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (i < k) {
          const T u = Ur[i * LDL + k];
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) x[cc][r] -= u * xk[cc];
        }
      }
    }
#pragma unroll
    for (int cc = 0; cc < 4; ++cc)
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (i < NB && j0 + cc < NB) Uout[i + (j0 + cc) * NB] = x[cc][r];
      }
  }
}

// Row interchanges of panels [p0, p0 + np) (in order) on the D columns
// [a0, a1) and [b0, b1) (clamped to the leaf) and, with with_x, on the
// leaf's X columns.  grid (column block, leaf); thread = column.
template <typename T>
__global__ void __launch_bounds__(kThreads)
    leaf_laswp_kernel(const LeafFactorTask<T> *__restrict__ tasks, int p0, int np, int nb,
                      int a0, int a1, int b0, int b1, int with_x) {
  const LeafFactorTask<T> tk = tasks[blockIdx.y];
  const int n = tk.n;
  if (p0 * nb >= n) return;
  bool any = false;
  for (int q = p0; q < p0 + np && q * nb < n; ++q) any |= tk.swapflag[q] != 0;
  if (!any) return;
  const int na = max(0, min(a1, n) - a0);
  const int nbr = max(0, min(b1, n) - b0);
  const int c = blockIdx.x * kThreads + threadIdx.x;
  T *col;
  if (c < na) {
    col = tk.D + (long long)(a0 + c) * tk.ldd;
  } else if (c < na + nbr) {
    col = tk.D + (long long)(b0 + c - na) * tk.ldd;
  } else if (with_x && c < na + nbr + tk.ncols) {
    col = tk.X + (long long)(c - na - nbr) * tk.ldx;
  } else {
    return;
  }
  for (int q = p0; q < p0 + np; ++q) {
    const int k0 = q * nb;
    if (k0 >= n) break;
    if (tk.swapflag[q] == 0) continue;
    const int kb = min(nb, n - k0);
    for (int j = 0; j < kb; ++j) {
      const int p = tk.ipiv[k0 + j] - 1;
      if (p != k0 + j) {
        const T t = col[k0 + j];
        col[k0 + j] = col[p];
        col[p] = t;
      }
    }
  }
}

template <typename T>
__global__ void leaf_init_kernel(const LeafFactorTask<T> *__restrict__ tasks, int *info) {
  const LeafFactorTask<T> tk = tasks[blockIdx.x];
  for (int i = threadIdx.x; i < tk.n; i += blockDim.x) tk.perm[i] = i;
  if (threadIdx.x == 0 && info) info[tk.info_slot] = 0;
}

// ---- apply: X <- U^{-1} L^{-1} P X with the stored blocked factors.
//
// One CTA per (column chunk of MC right-hand sides, leaf).  The chunk of P X
// lives in shared memory (row-major, padded rows); per panel the diagonal
// block is applied with its explicit inverse and the rest of the block
// column of L (forward) or U (backward) is streamed from global memory once,
// coalesced along the rows, into register accumulators.  Every element of the
// factors is read once per chunk.
constexpr int kApplyThreads = 512;


// Stage the diagonal-block inverse Ainv (kb x kb, column-major, ld nb) into
// shared memory `As` (ld kb + 1) with asynchronous copies (one commit group).
template <typename T>
__device__ inline void stage_inverse(const T *__restrict__ Ainv, int nb, int kb, T *As) {
  const int lds = kb + 1;
  for (int e = threadIdx.x; e < kb * kb; e += kApplyThreads) {
    const int i = e % kb, k = e / kb;
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(As + i + k * lds));
    if (sizeof(T) == 8)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(Ainv + i + (size_t)k * nb));
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(Ainv + i + (size_t)k * nb));
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// y (kb x MC in shared memory, row stride XS) <- As y, As the staged inverse.
template <typename T, int MC, int XS>
__device__ inline void apply_diag(T *y, int kb, const T *As) {
  constexpr int VW = 16 / sizeof(T);
  constexpr int NV = MC / VW;
  constexpr int OUT = (64 * NV + kApplyThreads - 1) / kApplyThreads;
  using V = typename Vec16<T>::V;
  const int tid = threadIdx.x;
  const int lds = kb + 1;
  T acc[OUT][VW];
#pragma unroll
  for (int o = 0; o < OUT; ++o) {
#pragma unroll
    for (int v = 0; v < VW; ++v) acc[o][v] = T(0);
    const int e = tid + o * kApplyThreads;
    if (e < kb * NV) {
      const int i = e % kb, jv = e / kb;
#pragma unroll 8
      for (int k = 0; k < kb; ++k) {
        const T a = As[i + k * lds];
        const V x = *reinterpret_cast<const V *>(y + k * XS + jv * VW);
        const T *xp = reinterpret_cast<const T *>(&x);
#pragma unroll
        for (int v = 0; v < VW; ++v) acc[o][v] += a * xp[v];
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int o = 0; o < OUT; ++o) {
    const int e = tid + o * kApplyThreads;
    if (e < kb * NV) {
      const int i = e % kb, jv = e / kb;
      V out;
      T *op = reinterpret_cast<T *>(&out);
#pragma unroll
      for (int v = 0; v < VW; ++v) op[v] = acc[o][v];
      *reinterpret_cast<V *>(y + i * XS + jv * VW) = out;
    }
  }
  __syncthreads();
}

// dst (rows x MC, shared, stride XS) -= A (rows x kb, global, ld lda) y (kb x MC, shared)
template <typename T, int MC, int XS>
__device__ inline void apply_block(const T *__restrict__ A, long long lda, T *dst, int rows,
                                   const T *y, int kb) {
  constexpr int VW = 16 / sizeof(T);
  using V = typename Vec16<T>::V;
  for (int i = threadIdx.x; i < rows; i += kApplyThreads) {
    T acc[MC];
#pragma unroll
    for (int j = 0; j < MC; j += VW) {
      const V x = *reinterpret_cast<const V *>(dst + i * XS + j);
      const T *xp = reinterpret_cast<const T *>(&x);
#pragma unroll
      for (int v = 0; v < VW; ++v) acc[j + v] = xp[v];
    }
    const T *Ai = A + i;
    constexpr int LB = sizeof(T) == 4 ? 64 : 32;  // loads in flight per row
    int k = 0;
    for (; k + LB <= kb; k += LB) {
      T a[LB];
#pragma unroll
      for (int u = 0; u < LB; ++u) a[u] = Ai[(long long)(k + u) * lda];
#pragma unroll
      for (int u = 0; u < LB; ++u) {
        const T *yk = y + (k + u) * XS;
#pragma unroll
        for (int j = 0; j < MC; j += VW) {
          const V x = *reinterpret_cast<const V *>(yk + j);
          const T *xp = reinterpret_cast<const T *>(&x);
#pragma unroll
          for (int v = 0; v < VW; ++v) acc[j + v] -= a[u] * xp[v];
        }
      }
    }
    for (; k < kb; ++k) {
      const T a = Ai[(long long)k * lda];
      const T *yk = y + k * XS;
#pragma unroll
      for (int j = 0; j < MC; ++j) acc[j] -= a * yk[j];
    }
#pragma unroll
    for (int j = 0; j < MC; j += VW) {
      V out;
      T *op = reinterpret_cast<T *>(&out);
#pragma unroll
      for (int v = 0; v < VW; ++v) op[v] = acc[j + v];
      *reinterpret_cast<V *>(dst + i * XS + j) = out;
    }
  }
}

template <typename T, int MC>
__global__ void __launch_bounds__(kApplyThreads)
    leaf_apply_kernel(const LeafFactorTask<T> *__restrict__ tasks, int nb, int max_n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int XS = MC + 16 / sizeof(T);  // padded row stride (16 bytes)
  const LeafFactorTask<T> tk = tasks[blockIdx.y];
  const int n = tk.n;
  const int c0 = blockIdx.x * MC;
  if (c0 >= tk.ncols || n <= 0) return;
  const int mc = min(MC, tk.ncols - c0);
  const int tid = threadIdx.x;
  T *xs = reinterpret_cast<T *>(smem_raw);
  T *As0 = xs + (size_t)max_n * XS;  // two staged inverses, nb x (nb + 1) each
  const int as_stride = nb * (nb + 1);
  T *X = tk.X + (long long)c0 * tk.ldx;
  const long long ldx = tk.ldx, ldd = tk.ldd;
  const int np = (n + nb - 1) / nb;
  // step s < np: forward panel s with Linv_s; step s >= np: backward panel
  // 2 np - 1 - s with its Uinv.  The next step's inverse is staged while the
  // current one is applied.
  auto inv_of = [&](int st, int &k0, int &kb) -> const T * {
    const int p = st < np ? st : 2 * np - 1 - st;
    k0 = p * nb;
    kb = min(nb, n - k0);
    return (st < np ? tk.Linv : tk.Uinv) + (size_t)p * nb * nb;
  };
  {
    int k0, kb;
    const T *inv0 = inv_of(0, k0, kb);
    stage_inverse<T>(inv0, nb, kb, As0);
  }
  for (int e = tid; e < n * MC; e += kApplyThreads) {
    const int i = e % n, j = e / n;
    xs[i * XS + j] = j < mc ? X[tk.perm[i] + (long long)j * ldx] : T(0);
  }
  for (int st = 0; st < 2 * np; ++st) {
    int k0, kb;
    inv_of(st, k0, kb);
    if (st + 1 < 2 * np) {
      int k1, kb1;
      const T *inv1 = inv_of(st + 1, k1, kb1);
      stage_inverse<T>(inv1, nb, kb1, As0 + ((st + 1) & 1) * as_stride);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();  // this step's inverse and the previous step's updates visible
    apply_diag<T, MC, XS>(xs + k0 * XS, kb, As0 + (st & 1) * as_stride);
    if (st < np)
      apply_block<T, MC, XS>(tk.D + (k0 + kb) + (long long)k0 * ldd, ldd, xs + (k0 + kb) * XS,
                             n - k0 - kb, xs + k0 * XS, kb);
    else
      apply_block<T, MC, XS>(tk.D + (long long)k0 * ldd, ldd, xs, k0, xs + k0 * XS, kb);
    __syncthreads();
  }
  for (int e = tid; e < n * mc; e += kApplyThreads) {
    const int i = e % n, j = e / n;
    X[i + (long long)j * ldx] = xs[i * XS + j];
  }
}

// ---- inverses of the outer diagonal blocks (two-level factorization).
//
// For outer block J (rows / columns j0 .. j0 + obe of a leaf) with panels
// p = 0 .. P-1 of width NB, the unit-lower block inverse is built by block
// forward substitution from the panels' own inverses Linv_p:
//   X[p][p] = Linv_p,  X[p][q] = -Linv_p sum_{s=q}^{p-1} L[p][s] X[s][q]  (q < p),
// and the upper one by block back substitution from Uinv_p:
//   Y[p][p] = Uinv_p,  Y[q][p] = -Uinv_q sum_{s=q+1}^{p} U[q][s] Y[s][p]  (q < p).
// Lower: CTA (256 threads) = one leaf, for one block; upper: one leaf x one
// block, all blocks in one launch.  The ob x ob result, an NB x NB product
// tile and one staged NB x NB block of D live in shared memory (padded leading
// dimensions; the panel inverses are read from global memory), so two CTAs
// fit on an SM; products are 16 x 16 thread grids of R x R outputs.
constexpr int kInvThreads = 256;

template <typename T, int NB>
__device__ inline void tile_mm(const T *A, int lda, const T *B, int ldb, T *C, int ldc,
                               T alpha, bool acc) {
  constexpr int R = NB / 16;
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  T c[R][R];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int q = 0; q < R; ++q) c[r][q] = T(0);
#pragma unroll 4
  for (int k = 0; k < NB; ++k) {
    T a[R], b[R];
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = A[(ty * R + r) + k * lda];
#pragma unroll
    for (int q = 0; q < R; ++q) b[q] = B[k + (tx * R + q) * ldb];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if constexpr (sizeof(T) == 4 && R % 2 == 0) {
        // packed two-wide FMAs, each half rounded as c + a b
#pragma unroll
        for (int q = 0; q < R; q += 2) {
          const float2 v = __ffma2_rn(make_float2(a[r], a[r]), make_float2(b[q], b[q + 1]),
                                      make_float2(c[r][q], c[r][q + 1]));
          c[r][q] = v.x;
          c[r][q + 1] = v.y;
        }
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) c[r][q] += a[r] * b[q];
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int q = 0; q < R; ++q) {
      T *cp = C + (ty * R + r) + (tx * R + q) * ldc;
      *cp = (acc ? *cp : T(0)) + alpha * c[r][q];
    }
}

template <typename T, int NB>
__global__ void __launch_bounds__(kInvThreads)
    leaf_block_inverse_kernel(const LeafFactorTask<T> *__restrict__ tasks, int ob, int J0,
                              int upper) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const LeafFactorTask<T> tk = tasks[blockIdx.x];
  const int n = tk.n;
  const int J = upper ? (int)blockIdx.y : J0;  // upper: every block, one per grid row
  const int j0 = J * ob;
  if (j0 >= n) return;
  const int obe = min(ob, n - j0);
  const int P = (obe + NB - 1) / NB;
  const int pbase = j0 / NB;
  constexpr int LT = NB + 1;  // padded ld of the NB x NB tiles
  const int LX = ob + 1;      // padded ld of the block inverse
  T *X = reinterpret_cast<T *>(smem_raw);  // ob x ob
  T *Tt = X + (size_t)ob * LX;             // product tile
  T *Bs = Tt + NB * LT;                    // staged L / U block of D
  const int tid = threadIdx.x;
  for (int e = tid; e < ob * ob; e += kInvThreads) X[(e % ob) + (e / ob) * LX] = T(0);
  // panel pi's inverse (NB x NB, ld NB; identity beyond the leaf), read from
  // global memory (L1 / L2) by the products
  auto inv_of = [&](int pi) { return (upper ? tk.Uinv : tk.Linv) + (size_t)pi * NB * NB; };
  // stage the NB x NB block of D at block panels (pr, pc), zero outside the block
  auto stage_d = [&](int pr, int pc) {
    for (int e = tid; e < NB * NB; e += kInvThreads) {
      const int i = e % NB, c = e / NB;
      const int gi = pr * NB + i, gc = pc * NB + c;
      Bs[i + c * LT] = (gi < obe && gc < obe) ? tk.D[(j0 + gi) + (long long)(j0 + gc) * tk.ldd] : T(0);
    }
  };
  auto Xb = [&](int pr, int pc) { return X + pr * NB + (size_t)pc * NB * LX; };
  for (int p = 0; p < P; ++p) {
    __syncthreads();
    {
      const T *src = inv_of(pbase + p);
      for (int e = tid; e < NB * NB; e += kInvThreads) {
        const int i = e % NB, c = e / NB;
        Xb(p, p)[i + c * LX] = src[e];
      }
    }
    if (!upper) {
      for (int q = 0; q < p; ++q) {
        // Tt = sum_{s=q}^{p-1} L[p][s] X[s][q];  X[p][q] = -Linv_p Tt
        for (int s2 = q; s2 < p; ++s2) {
          __syncthreads();
          stage_d(p, s2);
          __syncthreads();
          tile_mm<T, NB>(Bs, LT, Xb(s2, q), LX, Tt, LT, T(1), s2 > q);
        }
        __syncthreads();
        tile_mm<T, NB>(inv_of(pbase + p), NB, Tt, LT, Xb(p, q), LX, T(-1), false);
      }
    } else {
      for (int q = p - 1; q >= 0; --q) {
        // Tt = sum_{s=q+1}^{p} U[q][s] Y[s][p];  Y[q][p] = -Uinv_q Tt
        for (int s2 = q + 1; s2 <= p; ++s2) {
          __syncthreads();
          stage_d(q, s2);
          __syncthreads();
          tile_mm<T, NB>(Bs, LT, Xb(s2, p), LX, Tt, LT, T(1), s2 > q + 1);
        }
        __syncthreads();
        tile_mm<T, NB>(inv_of(pbase + q), NB, Tt, LT, Xb(q, p), LX, T(-1), false);
      }
    }
  }
  __syncthreads();
  // zero outside the leaf's part of the block (rows / columns >= obe)
  T *dst = (upper ? tk.UinvB : tk.LinvB) + (size_t)J * ob * ob;
  for (int e = tid; e < ob * ob; e += kInvThreads) {
    const int i = e % ob, c = e / ob;
    dst[e] = (i < obe && c < obe) ? X[i + c * LX] : T(0);
  }
}

}  // namespace

template <int NB, typename T>
size_t panel_smem(int ps) {
  return (size_t)ps * NB * sizeof(T) + 2 * (size_t)NB * NB * sizeof(T) + 2 * NB * sizeof(int) +
         16 * sizeof(T) + 32 * sizeof(int) + (size_t)ps * sizeof(int) + 64;
}

template <typename T>
void launch_leaf_init(const LeafFactorTask<T> *tasks, int count, int *info, cudaStream_t s) {
  if (count <= 0) return;
  leaf_init_kernel<T><<<count, kThreads, 0, s>>>(tasks, info);
  HODLR_LAUNCH_CHECK();
}

template <typename T, int NB>
void launch_leaf_panel_nb(const LeafFactorTask<T> *tasks, int count, int max_n, int k0,
                          int panel, int *info, cudaStream_t s) {
  const int ps = (max_n - k0 + 3) & ~3;
  // the panel buffer doubles as the inverses' output (2 NB^2 elements)
  const int psz = ps < 2 * NB ? 2 * NB : ps;
  const size_t smem = panel_smem<NB, T>(psz);
  raise_smem_limit(reinterpret_cast<const void *>(leaf_panel_kernel<T, NB>), smem);
  leaf_panel_kernel<T, NB><<<count, kThreads, smem, s>>>(tasks, k0, panel, psz, info);
  HODLR_LAUNCH_CHECK();
}

template <typename T, int NB, int RPT>
void launch_leaf_panel_reg(const LeafFactorTask<T> *tasks, int count, int rows, int k0,
                           int panel, int *info, cudaStream_t s) {
  // one warp per 32 x RPT live rows of the largest leaf's panel
  const int threads = std::min(kRegThreads, std::max(32, cdiv(cdiv(rows, RPT), 32) * 32));
  leaf_panel_reg_kernel<T, NB, RPT><<<count, threads, 0, s>>>(tasks, k0, panel, info);
  HODLR_LAUNCH_CHECK();
}

template <typename T>
void launch_leaf_panel(const LeafFactorTask<T> *tasks, int count, int max_n, int nb, int k0,
                       int panel, int *info, cudaStream_t s) {
  if (count <= 0) return;
  // register-resident panel: rows <= 512 RPT with 64 values per thread
  const int rows = max_n - k0;
  if constexpr (sizeof(T) == 4) {
    if (nb == 64 && rows <= kRegThreads)
      return launch_leaf_panel_reg<T, 64, 1>(tasks, count, rows, k0, panel, info, s);
    if (nb == 32 && rows <= 2 * kRegThreads)
      return launch_leaf_panel_reg<T, 32, 2>(tasks, count, rows, k0, panel, info, s);
  } else {
    if (nb == 32 && rows <= kRegThreads)
      return launch_leaf_panel_reg<T, 32, 1>(tasks, count, rows, k0, panel, info, s);
    if (nb == 16 && rows <= 2 * kRegThreads)
      return launch_leaf_panel_reg<T, 16, 2>(tasks, count, rows, k0, panel, info, s);
  }
  if (sizeof(T) == 8) {
    if (nb == 32) launch_leaf_panel_nb<T, 32>(tasks, count, max_n, k0, panel, info, s);
    else launch_leaf_panel_nb<T, 16>(tasks, count, max_n, k0, panel, info, s);
  } else {
    if (nb == 64) launch_leaf_panel_nb<T, 64>(tasks, count, max_n, k0, panel, info, s);
    else launch_leaf_panel_nb<T, 32>(tasks, count, max_n, k0, panel, info, s);
  }
}

template <typename T>
void launch_leaf_laswp(const LeafFactorTask<T> *tasks, int count, int max_cols, int nb, int p0,
                       int np, int a0, int a1, int b0, int b1, bool with_x, cudaStream_t s) {
  if (count <= 0 || max_cols <= 0 || np <= 0) return;
  dim3 grid(cdiv(max_cols, kThreads), count);
  leaf_laswp_kernel<T><<<grid, kThreads, 0, s>>>(tasks, p0, np, nb, a0, a1, b0, b1,
                                                 with_x ? 1 : 0);
  HODLR_LAUNCH_CHECK();
}

template <typename T, int MC>
void launch_leaf_apply_mc(const LeafFactorTask<T> *tasks, int count, int max_n, int max_cols,
                          int nb, cudaStream_t s) {
  constexpr int XS = MC + 16 / sizeof(T);
  const size_t smem = ((size_t)max_n * XS + 2 * (size_t)nb * (nb + 1)) * sizeof(T);
  raise_smem_limit(reinterpret_cast<const void *>(leaf_apply_kernel<T, MC>), smem);
  dim3 grid(cdiv(max_cols, MC), count);
  leaf_apply_kernel<T, MC><<<grid, kApplyThreads, smem, s>>>(tasks, nb, max_n);
  HODLR_LAUNCH_CHECK();
}

template <typename T>
void launch_leaf_apply(const LeafFactorTask<T> *tasks, int count, int max_n, int max_cols, int nb,
                       cudaStream_t s) {
  if (count <= 0 || max_cols <= 0 || max_n <= 0) return;
  if (nb > 64) throw CudaError{cudaErrorInvalidValue};
  // the chunk of P X is max_n x (MC + pad) in shared memory (<= 160 KB)
  const bool wide_ok = ((size_t)max_n * (32 + 16 / sizeof(T)) + 2 * (size_t)nb * (nb + 1)) *
                           sizeof(T) <= 180 * 1024;
  if (max_cols <= 8) launch_leaf_apply_mc<T, 8>(tasks, count, max_n, max_cols, nb, s);
  else if (max_cols <= 16 || !wide_ok) launch_leaf_apply_mc<T, 16>(tasks, count, max_n, max_cols, nb, s);
  else launch_leaf_apply_mc<T, 32>(tasks, count, max_n, max_cols, nb, s);
}

template <typename T>
void launch_leaf_block_inverse(const LeafFactorTask<T> *tasks, int count, int nb, int ob, int J,
                               bool upper, int nblocks, cudaStream_t s) {
  if (count <= 0 || (upper && nblocks <= 0)) return;
  if (ob > 128 || ob % nb) throw CudaError{cudaErrorInvalidValue};
  dim3 grid(count, upper ? nblocks : 1);
  auto go = [&](auto kern, int NBv) {
    const size_t smem = ((size_t)ob * (ob + 1) + 2 * (size_t)NBv * (NBv + 1)) * sizeof(T);
    raise_smem_limit(reinterpret_cast<const void *>(kern), smem);
    kern<<<grid, kInvThreads, smem, s>>>(tasks, ob, J, upper ? 1 : 0);
  };
  if (nb == 64) go(leaf_block_inverse_kernel<T, 64>, 64);
  else if (nb == 32) go(leaf_block_inverse_kernel<T, 32>, 32);
  else if (nb == 16) go(leaf_block_inverse_kernel<T, 16>, 16);
  else throw CudaError{cudaErrorInvalidValue};
  HODLR_LAUNCH_CHECK();
}

template void launch_leaf_block_inverse<double>(const LeafFactorTask<double> *, int, int, int,
                                                int, bool, int, cudaStream_t);
template void launch_leaf_block_inverse<float>(const LeafFactorTask<float> *, int, int, int, int,
                                               bool, int, cudaStream_t);

template void launch_leaf_apply<double>(const LeafFactorTask<double> *, int, int, int, int,
                                        cudaStream_t);
template void launch_leaf_apply<float>(const LeafFactorTask<float> *, int, int, int, int,
                                       cudaStream_t);
template void launch_leaf_init<double>(const LeafFactorTask<double> *, int, int *, cudaStream_t);
template void launch_leaf_init<float>(const LeafFactorTask<float> *, int, int *, cudaStream_t);
template void launch_leaf_panel<double>(const LeafFactorTask<double> *, int, int, int, int, int,
                                        int *, cudaStream_t);
template void launch_leaf_panel<float>(const LeafFactorTask<float> *, int, int, int, int, int,
                                       int *, cudaStream_t);
template void launch_leaf_laswp<double>(const LeafFactorTask<double> *, int, int, int, int, int,
                                        int, int, int, int, bool, cudaStream_t);
template void launch_leaf_laswp<float>(const LeafFactorTask<float> *, int, int, int, int, int,
                                       int, int, int, int, bool, cudaStream_t);

}  // namespace hodlr
