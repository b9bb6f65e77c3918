// leaf.cu -- batched leaf solve: LU with partial pivoting + triangular solves.
//
// GPU restatement of the leaf task body of fastSolver
// (src/solver/solver_tasks.cc:424-450: dgesv(D_leaf, [b | U_anc])).  Two
// kernels, each batched over every leaf of a launch:
//
//   getrf_kernel  one CTA per leaf.  Right-looking blocked LU: the current
//                 panel (rows k0..n, PW columns) is factored in shared memory
//                 (argmax pivot with lowest-index tie break, as LAPACK's
//                 idamax), written back, and the trailing columns are updated
//                 tile by tile: row interchanges, U12 = L11^{-1} A12 and
//                 A22 -= L21 U12 with register-tiled FMAs.  Interchanges are
//                 also applied to the columns left of the panel, so D ends in
//                 LAPACK dgetrf layout.  The final row order is kept as
//                 `perm` for the solve.
//   getrs_kernel  grid (column tile, leaf).  The tile of X (all n rows, W
//                 columns) is gathered through `perm` into shared memory, then
//                 forward (unit L) and backward (U) substitution run in blocks
//                 of BK rows: a diagonal-block triangle per column followed by
//                 a rank-BK update of the remaining rows, one thread per row
//                 with W accumulators and L/U streamed from L2.
//
// T = double for the FP64 path, float for the mixed path's FP32 factor.
#include "common.cuh"
#include "leaf.cuh"

namespace hodlr {

namespace {

constexpr int kGetrfThreads = 256;
constexpr int kTileCols = 64;  // trailing-update column tile

template <typename T>
__device__ inline T tabs(T v) {
  return v < T(0) ? -v : v;
}

// ---------------------------------------------------------------------------
// getrf
// ---------------------------------------------------------------------------

template <typename T, int PW>
__global__ void __launch_bounds__(kGetrfThreads)
    getrf_kernel(const LeafTask<T> *tasks, LeafTask<T> single, int *info,
                 int panel_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const LeafTask<T> tk = tasks ? tasks[blockIdx.x] : single;
  const int n = tk.n;
  if (n <= 0) return;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  T *D = tk.D;
  const long long ldd = tk.ldd;

  const int PS = panel_stride;             // >= n, panel column stride
  T *P = reinterpret_cast<T *>(smem_raw);  // PS x PW
  T *Us = P + (size_t)PS * PW;             // PW x kTileCols (row k stride kTileCols)
  int *perm = reinterpret_cast<int *>(Us + PW * kTileCols);  // n
  int *pv = perm + PS;                                         // PW: panel pivots (relative)
  T *redv = reinterpret_cast<T *>(pv + PW + (PW & 1));         // 8
  int *redi = reinterpret_cast<int *>(redv + 8);               // 8
  __shared__ int s_info;

  for (int i = tid; i < n; i += kGetrfThreads) perm[i] = i;
  if (tid == 0) s_info = 0;
  __syncthreads();

  for (int k0 = 0; k0 < n; k0 += PW) {
    const int kb = min(PW, n - k0);
    const int R = n - k0;
    // ---- load panel rows k0..n-1, columns k0..k0+kb-1
    for (int j = 0; j < kb; ++j) {
      const T *src = D + (k0 + j) * ldd + k0;
      for (int i = tid; i < R; i += kGetrfThreads) P[i + (size_t)j * PS] = src[i];
    }
    __syncthreads();
    // ---- unblocked LU of the panel in shared memory
    for (int j = 0; j < kb; ++j) {
      T best = T(-1);
      int bi = R;
      for (int i = j + tid; i < R; i += kGetrfThreads) {
        T a = tabs(P[i + (size_t)j * PS]);
        if (a > best) { best = a; bi = i; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        T ob = __shfl_down_sync(0xffffffffu, best, off);
        int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) { redv[warp] = best; redi[warp] = bi; }
      __syncthreads();
      if (tid == 0) {
        T b = redv[0];
        int ii = redi[0];
        for (int w = 1; w < kGetrfThreads / 32; ++w)
          if (redv[w] > b || (redv[w] == b && redi[w] < ii)) { b = redv[w]; ii = redi[w]; }
        if (ii >= R) ii = j;  // all-NaN column: keep the diagonal
        pv[j] = ii;
        if (tk.ipiv) tk.ipiv[k0 + j] = k0 + ii + 1;
        if (ii != j) {
          int t = perm[k0 + j]; perm[k0 + j] = perm[k0 + ii]; perm[k0 + ii] = t;
        }
        if (P[ii + (size_t)j * PS] == T(0) && s_info == 0) s_info = k0 + j + 1;
      }
      __syncthreads();
      const int p = pv[j];
      if (p != j) {
        for (int c = tid; c < kb; c += kGetrfThreads) {
          T t = P[j + (size_t)c * PS];
          P[j + (size_t)c * PS] = P[p + (size_t)c * PS];
          P[p + (size_t)c * PS] = t;
        }
        __syncthreads();
      }
      const T piv = P[j + (size_t)j * PS];
      if (piv != T(0)) {
        const T rinv = T(1) / piv;
        for (int i = j + 1 + tid; i < R; i += kGetrfThreads) {
          T l = P[i + (size_t)j * PS] * rinv;
          P[i + (size_t)j * PS] = l;
          for (int c = j + 1; c < kb; ++c) P[i + (size_t)c * PS] -= l * P[j + (size_t)c * PS];
        }
      }
      __syncthreads();
    }
    // ---- write the factored panel back
    for (int j = 0; j < kb; ++j) {
      T *dst = D + (k0 + j) * ldd + k0;
      for (int i = tid; i < R; i += kGetrfThreads) dst[i] = P[i + (size_t)j * PS];
    }
    // ---- interchanges on the columns left of the panel (LAPACK layout)
    for (int j = 0; j < kb; ++j) {
      const int p = pv[j];
      if (p != j) {
        for (int c = tid; c < k0; c += kGetrfThreads) {
          T *col = D + (long long)c * ldd;
          T t = col[k0 + j]; col[k0 + j] = col[k0 + p]; col[k0 + p] = t;
        }
      }
    }
    // ---- trailing update, one column tile at a time
    const int R2 = R - kb;  // rows below the panel
    for (int c0 = k0 + kb; c0 < n; c0 += kTileCols) {
      const int nc = min(kTileCols, n - c0);
      // (1) top kb rows of the tile into Us with the panel's interchanges
      if (tid < nc) {
        T *col = D + (long long)(c0 + tid) * ldd;
        for (int j = 0; j < kb; ++j) Us[j * kTileCols + tid] = col[k0 + j];
        for (int j = 0; j < kb; ++j) {
          const int p = pv[j];
          if (p != j) {
            if (p < kb) {
              T t = Us[j * kTileCols + tid];
              Us[j * kTileCols + tid] = Us[p * kTileCols + tid];
              Us[p * kTileCols + tid] = t;
            } else {
              T t = Us[j * kTileCols + tid];
              Us[j * kTileCols + tid] = col[k0 + p];
              col[k0 + p] = t;
            }
          }
        }
        // (2) U12 = L11^{-1} A12 (unit lower), one column per thread
        for (int i = 1; i < kb; ++i) {
          T s = Us[i * kTileCols + tid];
          for (int k = 0; k < i; ++k) s -= P[i + (size_t)k * PS] * Us[k * kTileCols + tid];
          Us[i * kTileCols + tid] = s;
        }
        for (int j = 0; j < kb; ++j) col[k0 + j] = Us[j * kTileCols + tid];
      }
      __syncthreads();
      // (3) A22 -= L21 * U12, 128 x 64 per pass, 4 x 8 per thread
      const int lr = lane & 7, lc = lane >> 3;
      const int wr = warp & 3, wc = warp >> 2;
      const int row_in = wr * 32 + lr * 4;  // within the 128-row pass
      const int col_in = wc * 32 + lc * 8;  // within the tile
      for (int rb = 0; rb < R2; rb += 128) {
        T acc[4][8];
        const int r_loc = kb + rb + row_in;  // relative to k0
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          const int cc = col_in + b;
          T *col = D + (long long)(c0 + cc) * ldd + k0;
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int rr = r_loc + a;
            acc[a][b] = (cc < nc && rr < R) ? col[rr] : T(0);
          }
        }
        for (int k = 0; k < kb; ++k) {
          T av[4], bv[8];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int rr = r_loc + a;
            av[a] = rr < R ? P[rr + (size_t)k * PS] : T(0);
          }
#pragma unroll
          for (int b = 0; b < 8; ++b) bv[b] = Us[k * kTileCols + col_in + b];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] -= av[a] * bv[b];
        }
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          const int cc = col_in + b;
          if (cc >= nc) continue;
          T *col = D + (long long)(c0 + cc) * ldd + k0;
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int rr = r_loc + a;
            if (rr < R) col[rr] = acc[a][b];
          }
        }
      }
      __syncthreads();
    }
    __syncthreads();
  }
  if (tk.perm)
    for (int i = tid; i < n; i += kGetrfThreads) tk.perm[i] = perm[i];
  if (tid == 0 && info) info[tk.info_slot] = s_info;
}

// ---------------------------------------------------------------------------
// getrs
// ---------------------------------------------------------------------------

constexpr int kGetrsThreads = 256;
constexpr int kBK = 32;

template <typename T, int W>
__global__ void __launch_bounds__(kGetrsThreads)
    getrs_kernel(const LeafTask<T> *tasks, LeafTask<T> single) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const LeafTask<T> tk = tasks ? tasks[blockIdx.y] : single;
  const int n = tk.n;
  const int c0 = blockIdx.x * W;
  if (n <= 0 || c0 >= tk.nrhs) return;
  const int nc = min(W, tk.nrhs - c0);
  const int tid = threadIdx.x;
  constexpr int XS = W + 2;  // padded row stride of the tile
  T *Xs = reinterpret_cast<T *>(smem_raw);        // n x XS (row-major)
  T *Ls = Xs + (size_t)n * XS;                    // kBK x kBK diagonal block
  int *sperm = reinterpret_cast<int *>(Ls + kBK * kBK);  // n
  const T *D = tk.D;
  const long long ldd = tk.ldd;
  T *X = tk.X;
  const long long ldx = tk.ldx;
  const int *perm = tk.perm;
  if (!perm && tk.ipiv) {
    // row order from LAPACK pivots: apply the interchanges to 0..n-1
    for (int i = tid; i < n; i += kGetrsThreads) sperm[i] = i;
    __syncthreads();
    if (tid == 0)
      for (int j = 0; j < n; ++j) {
        const int p = tk.ipiv[j] - 1;
        if (p != j) { int t = sperm[j]; sperm[j] = sperm[p]; sperm[p] = t; }
      }
    __syncthreads();
    perm = sperm;
  }

  // gather the tile through the row permutation
  for (int c = 0; c < W; ++c) {
    const T *src = X + (long long)(c0 + c) * ldx;
    for (int i = tid; i < n; i += kGetrsThreads)
      Xs[i * XS + c] = (c < nc) ? src[perm ? perm[i] : i] : T(0);
  }
  __syncthreads();

  // ---- forward substitution, unit lower L
  for (int k0 = 0; k0 < n; k0 += kBK) {
    const int kb = min(kBK, n - k0);
    for (int e = tid; e < kb * kb; e += kGetrsThreads) {
      const int i = e % kb, k = e / kb;
      Ls[i + k * kBK] = D[(k0 + i) + (long long)(k0 + k) * ldd];
    }
    __syncthreads();
    if (tid < W) {
      for (int i = 1; i < kb; ++i) {
        T s = Xs[(k0 + i) * XS + tid];
        for (int k = 0; k < i; ++k) s -= Ls[i + k * kBK] * Xs[(k0 + k) * XS + tid];
        Xs[(k0 + i) * XS + tid] = s;
      }
    }
    __syncthreads();
    for (int row = k0 + kb + tid; row < n; row += kGetrsThreads) {
      T acc[W];
#pragma unroll
      for (int c = 0; c < W; ++c) acc[c] = Xs[row * XS + c];
      const T *lrow = D + row + (long long)k0 * ldd;
#pragma unroll 4
      for (int k = 0; k < kb; ++k) {
        const T l = lrow[(long long)k * ldd];
#pragma unroll
        for (int c = 0; c < W; ++c) acc[c] -= l * Xs[(k0 + k) * XS + c];
      }
#pragma unroll
      for (int c = 0; c < W; ++c) Xs[row * XS + c] = acc[c];
    }
    __syncthreads();
  }
  // ---- backward substitution, upper U
  for (int k1 = n; k1 > 0; k1 -= kBK) {
    const int k0 = max(0, k1 - kBK);
    const int kb = k1 - k0;
    for (int e = tid; e < kb * kb; e += kGetrsThreads) {
      const int i = e % kb, k = e / kb;
      Ls[i + k * kBK] = D[(k0 + i) + (long long)(k0 + k) * ldd];
    }
    __syncthreads();
    if (tid < W) {
      for (int i = kb - 1; i >= 0; --i) {
        T s = Xs[(k0 + i) * XS + tid];
        for (int k = i + 1; k < kb; ++k) s -= Ls[i + k * kBK] * Xs[(k0 + k) * XS + tid];
        Xs[(k0 + i) * XS + tid] = s / Ls[i + i * kBK];
      }
    }
    __syncthreads();
    for (int row = tid; row < k0; row += kGetrsThreads) {
      T acc[W];
#pragma unroll
      for (int c = 0; c < W; ++c) acc[c] = Xs[row * XS + c];
      const T *urow = D + row + (long long)k0 * ldd;
#pragma unroll 4
      for (int k = 0; k < kb; ++k) {
        const T u = urow[(long long)k * ldd];
#pragma unroll
        for (int c = 0; c < W; ++c) acc[c] -= u * Xs[(k0 + k) * XS + c];
      }
#pragma unroll
      for (int c = 0; c < W; ++c) Xs[row * XS + c] = acc[c];
    }
    __syncthreads();
  }
  for (int c = 0; c < nc; ++c) {
    T *dst = X + (long long)(c0 + c) * ldx;
    for (int i = tid; i < n; i += kGetrsThreads) dst[i] = Xs[i * XS + c];
  }
}

template <typename T>
constexpr int panel_width(int max_n) {
  return sizeof(T) == 8 ? (max_n <= 512 ? 32 : 16) : (max_n <= 512 ? 64 : 32);
}

template <typename T, int PW>
size_t getrf_smem(int ps) {
  return (size_t)ps * PW * sizeof(T) + (size_t)PW * kTileCols * sizeof(T) +
         (size_t)(ps + PW + 2) * sizeof(int) + 8 * sizeof(T) + 8 * sizeof(int) + 64;
}

template <typename T, int PW>
void launch_getrf_pw(const LeafTask<T> *tasks, const LeafTask<T> &single, int count,
                     int max_n, int *info, cudaStream_t s) {
  const int ps = (max_n + 3) & ~3;
  const size_t smem = getrf_smem<T, PW>(ps);
  raise_smem_limit(reinterpret_cast<const void *>(getrf_kernel<T, PW>), smem);
  getrf_kernel<T, PW><<<count, kGetrfThreads, smem, s>>>(tasks, single, info, ps);
  HODLR_LAUNCH_CHECK();
}

template <typename T>
int getrs_width() {
  return sizeof(T) == 8 ? 16 : 32;
}

template <typename T, int W>
void launch_getrs_w(const LeafTask<T> *tasks, const LeafTask<T> &single, int count,
                    int max_n, int max_nrhs, cudaStream_t s) {
  const size_t smem =
      (size_t)max_n * (W + 2) * sizeof(T) + kBK * kBK * sizeof(T) + (size_t)max_n * sizeof(int);
  raise_smem_limit(reinterpret_cast<const void *>(getrs_kernel<T, W>), smem);
  dim3 grid(cdiv(max_nrhs, W), count);
  getrs_kernel<T, W><<<grid, kGetrsThreads, smem, s>>>(tasks, single);
  HODLR_LAUNCH_CHECK();
}

}  // namespace

template <typename T>
void launch_getrf(const LeafTask<T> *tasks, const LeafTask<T> &single, int count,
                  int max_n, int *info, cudaStream_t s) {
  if (count <= 0 || max_n <= 0) return;
  const int pw = panel_width<T>(max_n);
  if (sizeof(T) == 8) {
    if (pw == 32) launch_getrf_pw<T, 32>(tasks, single, count, max_n, info, s);
    else launch_getrf_pw<T, 16>(tasks, single, count, max_n, info, s);
  } else {
    if (pw == 64) launch_getrf_pw<T, 64>(tasks, single, count, max_n, info, s);
    else launch_getrf_pw<T, 32>(tasks, single, count, max_n, info, s);
  }
}

template <typename T>
void launch_getrs(const LeafTask<T> *tasks, const LeafTask<T> &single, int count,
                  int max_n, int max_nrhs, cudaStream_t s) {
  if (count <= 0 || max_n <= 0 || max_nrhs <= 0) return;
  if (sizeof(T) == 8) launch_getrs_w<T, 16>(tasks, single, count, max_n, max_nrhs, s);
  else launch_getrs_w<T, 32>(tasks, single, count, max_n, max_nrhs, s);
}

template void launch_getrf<double>(const LeafTask<double> *, const LeafTask<double> &, int,
                                   int, int *, cudaStream_t);
template void launch_getrf<float>(const LeafTask<float> *, const LeafTask<float> &, int, int,
                                  int *, cudaStream_t);
template void launch_getrs<double>(const LeafTask<double> *, const LeafTask<double> &, int,
                                   int, int, cudaStream_t);
template void launch_getrs<float>(const LeafTask<float> *, const LeafTask<float> &, int, int,
                                  int, cudaStream_t);

}  // namespace hodlr
