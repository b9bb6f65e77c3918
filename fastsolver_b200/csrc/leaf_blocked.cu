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
#include "common.cuh"
#include "leaf_blocked.cuh"

namespace hodlr {

namespace {

constexpr int kThreads = 256;

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

// Row interchanges of panel `panel` on every column of D outside the panel
// and on the leaf's X columns.  grid (column block, leaf); thread = column.
template <typename T>
__global__ void __launch_bounds__(kThreads)
    leaf_laswp_kernel(const LeafFactorTask<T> *__restrict__ tasks, int k0, int panel, int nb) {
  const LeafFactorTask<T> tk = tasks[blockIdx.y];
  const int n = tk.n;
  if (k0 >= n || tk.swapflag[panel] == 0) return;
  const int kb = min(nb, n - k0);
  const int c = blockIdx.x * kThreads + threadIdx.x;
  const int nd = n - kb;  // D columns outside the panel
  T *col;
  if (c < nd) {
    const int dc = c < k0 ? c : c + kb;
    col = tk.D + (long long)dc * tk.ldd;
  } else if (c < nd + tk.ncols) {
    col = tk.X + (long long)(c - nd) * tk.ldx;
  } else {
    return;
  }
  for (int j = 0; j < kb; ++j) {
    const int p = tk.ipiv[k0 + j] - 1;
    if (p != k0 + j) {
      const T t = col[k0 + j];
      col[k0 + j] = col[p];
      col[p] = t;
    }
  }
}

template <typename T>
__global__ void leaf_init_kernel(const LeafFactorTask<T> *__restrict__ tasks, int *info) {
  const LeafFactorTask<T> tk = tasks[blockIdx.x];
  for (int i = threadIdx.x; i < tk.n; i += blockDim.x) tk.perm[i] = i;
  if (threadIdx.x == 0 && info) info[tk.info_slot] = 0;
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
  HODLR_CUDA_TRY(cudaFuncSetAttribute(leaf_panel_kernel<T, NB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  leaf_panel_kernel<T, NB><<<count, kThreads, smem, s>>>(tasks, k0, panel, psz, info);
  HODLR_LAUNCH_CHECK();
}

template <typename T>
void launch_leaf_panel(const LeafFactorTask<T> *tasks, int count, int max_n, int nb, int k0,
                       int panel, int *info, cudaStream_t s) {
  if (count <= 0) return;
  if (sizeof(T) == 8) {
    if (nb == 32) launch_leaf_panel_nb<T, 32>(tasks, count, max_n, k0, panel, info, s);
    else launch_leaf_panel_nb<T, 16>(tasks, count, max_n, k0, panel, info, s);
  } else {
    if (nb == 64) launch_leaf_panel_nb<T, 64>(tasks, count, max_n, k0, panel, info, s);
    else launch_leaf_panel_nb<T, 32>(tasks, count, max_n, k0, panel, info, s);
  }
}

template <typename T>
void launch_leaf_laswp(const LeafFactorTask<T> *tasks, int count, int max_cols, int nb, int k0,
                       int panel, cudaStream_t s) {
  if (count <= 0 || max_cols <= 0) return;
  dim3 grid(cdiv(max_cols, kThreads), count);
  leaf_laswp_kernel<T><<<grid, kThreads, 0, s>>>(tasks, k0, panel, nb);
  HODLR_LAUNCH_CHECK();
}

template void launch_leaf_init<double>(const LeafFactorTask<double> *, int, int *, cudaStream_t);
template void launch_leaf_init<float>(const LeafFactorTask<float> *, int, int *, cudaStream_t);
template void launch_leaf_panel<double>(const LeafFactorTask<double> *, int, int, int, int, int,
                                        int *, cudaStream_t);
template void launch_leaf_panel<float>(const LeafFactorTask<float> *, int, int, int, int, int,
                                       int *, cudaStream_t);
template void launch_leaf_laswp<double>(const LeafFactorTask<double> *, int, int, int, int, int,
                                        cudaStream_t);
template void launch_leaf_laswp<float>(const LeafFactorTask<float> *, int, int, int, int, int,
                                       cudaStream_t);

}  // namespace hodlr
