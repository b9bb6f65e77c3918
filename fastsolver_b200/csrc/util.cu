// util.cu -- element-wise kernels and device-side generators.
#include "common.cuh"
#include "util.cuh"

namespace hodlr {

namespace {

constexpr int kThreads = 256;

inline int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 64) b = 148LL * 64;
  return (int)(b > 0 ? b : 1);
}

// 4 consecutive rows of one column: dst = TD(src) or dst += TD(src); 16-byte
// vector accesses when `vec` (both column starts 16-byte aligned and all 4
// rows inside the matrix), else element by element.
template <typename T>
struct Vec4 {
  T v[4];
};
template <typename T>
__device__ inline Vec4<T> load4(const T *p) {
  Vec4<T> r;
  if constexpr (sizeof(T) == 4) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    r.v[0] = x.x; r.v[1] = x.y; r.v[2] = x.z; r.v[3] = x.w;
  } else {
    const double2 x = reinterpret_cast<const double2 *>(p)[0];
    const double2 y = reinterpret_cast<const double2 *>(p)[1];
    r.v[0] = x.x; r.v[1] = x.y; r.v[2] = y.x; r.v[3] = y.y;
  }
  return r;
}
template <typename T>
__device__ inline void store4(T *p, const Vec4<T> &r) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
  } else {
    reinterpret_cast<double2 *>(p)[0] = make_double2(r.v[0], r.v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(r.v[2], r.v[3]);
  }
}
template <typename TS, typename TD, bool ADD>
__device__ inline void move4(const TS *__restrict__ src, TD *__restrict__ dst, long long i,
                             long long rows, bool vec) {
  if (vec && i + 4 <= rows) {
    const Vec4<TS> x = load4(src + i);
    Vec4<TD> y;
    if (ADD) y = load4(dst + i);
#pragma unroll
    for (int u = 0; u < 4; ++u) y.v[u] = ADD ? TD(y.v[u] + TD(x.v[u])) : TD(x.v[u]);
    store4(dst + i, y);
  } else {
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (i + u < rows) {
        if (ADD) dst[i + u] += TD(src[i + u]);
        else dst[i + u] = TD(src[i + u]);
      }
  }
}

constexpr int kTileRows = 4 * kThreads;  // rows of one (column, tile) work unit

// dst (rows x cols, ldd) = TD(src) (or += with ADD): a grid-stride loop over
// (column, kTileRows-row tile) units, each thread moving 4 consecutive rows.
template <typename TS, typename TD, bool ADD>
__global__ void ew_tile_kernel(const TS *__restrict__ src, long long lds, TD *__restrict__ dst,
                               long long ldd, long long rows, long long cols, bool vec) {
  const long long rtiles = cdiv<long long>(rows, kTileRows);
  const long long total = rtiles * cols;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const long long j = t / rtiles;
    const long long i = (t - j * rtiles) * kTileRows + 4 * threadIdx.x;
    move4<TS, TD, ADD>(src + j * lds, dst + j * ldd, i, rows, vec);
  }
}

template <typename TS, typename TD>
bool vec_ok(const TS *src, long long lds, const TD *dst, long long ldd) {
  return (reinterpret_cast<uintptr_t>(src) % 16 == 0) && (reinterpret_cast<uintptr_t>(dst) % 16 == 0) &&
         (lds * (long long)sizeof(TS)) % 16 == 0 && (ldd * (long long)sizeof(TD)) % 16 == 0;
}

template <typename TS, typename TD, bool ADD>
void launch_ew_tile(const TS *src, long long lds, TD *dst, long long ldd, long long rows,
                    long long cols, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  const long long units = cdiv<long long>(rows, kTileRows) * cols;
  const unsigned grid = (unsigned)std::min<long long>(units, 148LL * 8);
  ew_tile_kernel<TS, TD, ADD><<<grid, kThreads, 0, s>>>(src, lds, dst, ldd, rows, cols,
                                                         vec_ok(src, lds, dst, ldd));
  HODLR_LAUNCH_CHECK();
}

// Sums of squares of r(:, c) and b(:, c) over one row chunk: CTA (c, chunk).
__global__ void colratio_part_kernel(const double *__restrict__ r, long long ldr,
                                     const double *__restrict__ b, long long ldb, long long rows,
                                     double *__restrict__ part) {
  __shared__ double sr[32], sb[32];
  const int c = blockIdx.x, q = blockIdx.y, nq = gridDim.y;
  const long long len = (rows + nq - 1) / nq;
  const long long i0 = q * len, i1 = min(rows, i0 + len);
  double ar = 0.0, ab = 0.0;
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const double x = r[i + c * ldr], y = b[i + c * ldb];
    ar += x * x;
    ab += y * y;
  }
  for (int off = 16; off > 0; off >>= 1) {
    ar += __shfl_down_sync(0xffffffffu, ar, off);
    ab += __shfl_down_sync(0xffffffffu, ab, off);
  }
  if ((threadIdx.x & 31) == 0) { sr[threadIdx.x >> 5] = ar; sb[threadIdx.x >> 5] = ab; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tr = 0.0, tb = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { tr += sr[w]; tb += sb[w]; }
    part[2 * ((long long)c * nq + q)] = tr;
    part[2 * ((long long)c * nq + q) + 1] = tb;
  }
}

// out[c] from the chunk sums, added in chunk order: one thread per column.
__global__ void colratio_fin_kernel(const double *__restrict__ part, int nq, int cols,
                                    double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double tr = 0.0, tb = 0.0;
  for (int q = 0; q < nq; ++q) {
    tr += part[2 * ((long long)c * nq + q)];
    tb += part[2 * ((long long)c * nq + q) + 1];
  }
  out[c] = tb > 0.0 ? sqrt(tr) / sqrt(tb) : sqrt(tr);
}


// Batched element-wise pass: one grid-stride loop over the tiles of all
// tasks (a tile = 1024 rows of one column; tile -> task by binary search on
// tile0), so large and small tasks share the grid evenly.  Each thread moves
// 4 rows of a tile, consecutive threads on consecutive rows.
template <typename TS, typename TD, bool ADD>
__global__ void ew2d_batched_kernel(const Ew2DTask<TS, TD> *__restrict__ tasks, int ntasks,
                                    long long total) {
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].tile0 <= t) lo = mid;
      else hi = mid - 1;
    }
    const Ew2DTask<TS, TD> &tk = tasks[lo];
    const long long rtiles = cdiv<long long>(tk.rows, kEwTileRows);
    const long long lt = t - tk.tile0;
    const long long j = lt / rtiles;
    const long long i0 = (lt - j * rtiles) * kEwTileRows;
    const bool vec = (reinterpret_cast<uintptr_t>(tk.src) % 16 == 0) &&
                     (reinterpret_cast<uintptr_t>(tk.dst) % 16 == 0) &&
                     (tk.lds * (long long)sizeof(TS)) % 16 == 0 &&
                     (tk.ldd * (long long)sizeof(TD)) % 16 == 0;
    move4<TS, TD, ADD>(tk.src + j * tk.lds, tk.dst + j * tk.ldd, i0 + 4 * threadIdx.x, tk.rows,
                       vec);
  }
}

// Batched column ratios (one CTA per column; batches supply many columns):
// blockIdx.y picks the system, blockIdx.x the column.
__global__ void colratio_batched_kernel(const RatioTask *__restrict__ tasks) {
  __shared__ double sr[32], sb[32];
  const RatioTask tk = tasks[blockIdx.y];
  const int c = blockIdx.x;
  if (c >= tk.cols) return;
  double ar = 0.0, ab = 0.0;
  for (long long i = threadIdx.x; i < tk.rows; i += blockDim.x) {
    const double x = tk.r[i + c * tk.ldr], y = tk.b[i + c * tk.ldb];
    ar += x * x;
    ab += y * y;
  }
  for (int off = 16; off > 0; off >>= 1) {
    ar += __shfl_down_sync(0xffffffffu, ar, off);
    ab += __shfl_down_sync(0xffffffffu, ab, off);
  }
  if ((threadIdx.x & 31) == 0) { sr[threadIdx.x >> 5] = ar; sb[threadIdx.x >> 5] = ab; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tr = 0.0, tb = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { tr += sr[w]; tb += sb[w]; }
    tk.out[c] = tb > 0.0 ? sqrt(tr) / sqrt(tb) : sqrt(tr);
  }
}

// dst[t][e] = sum_q src[t] + q * stride, fixed order (deterministic)
// (the slot values are loaded four at a time ahead of the adds, which keep
// the order q = 0, 1, 2, ...: the same sums)
template <typename T>
__global__ void sum_slots_kernel(const SumTask<T> *__restrict__ tasks) {
  const SumTask<T> tk = tasks[blockIdx.y];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tk.len;
       e += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    int q = 0;
    for (; q + 4 <= tk.nslots; q += 4) {
      T v[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) v[j] = tk.src[e + (q + j) * tk.stride];
#pragma unroll
      for (int j = 0; j < 4; ++j) acc += double(v[j]);
    }
    for (; q < tk.nslots; ++q) acc += double(tk.src[e + q * tk.stride]);
    tk.dst[e] = T(acc);
  }
}

__global__ void scale_cols_kernel(double *__restrict__ a, long long lda, long long rows,
                                  int cols, const double *__restrict__ s) {
  const long long total = rows * cols;
  const double f = *s;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % rows, j = e / rows;
    a[i + j * lda] *= f;
  }
}

// ----- generators ----------------------------------------------------------

// Reference test matrix: leaf block K = U U^T + diag I, U(i,j) = (g + i + j) % r
// with g the leaf's first global row (hodlr_matrix.cc:528-567).  Entries are
// exact integers (plus diag), so the result equals the reference's dgemm.
__global__ void circulant_k_kernel(const int2 *__restrict__ leaves, int nleaves, double *D,
                                   long long ldd, int r, double diag) {
  const int2 lf = leaves[blockIdx.y];  // (row_beg, nrow)
  const long long n = lf.y;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n * n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % n, j = e / n;
    const long long gi = lf.x + i, gj = lf.x + j;
    double acc = (i == j) ? diag : 0.0;
    for (int k = 0; k < r; ++k) acc += double((gi + k) % r) * double((gj + k) % r);
    D[lf.x + i + j * ldd] = acc;
  }
}

// U = V = (i + j) % r in global rows, every level block the same
// (init_matrix_tasks.cc:176-219 with the Hmat/U column layout).
__global__ void circulant_uv_kernel(double *U, long long ldu, double *V, long long ldv,
                                    long long N, int vcols, int r) {
  const long long total = N * vcols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % N;
    const int j = (int)(e / N);
    const double v = double((i + (j % r)) % r);
    U[i + j * ldu] = v;
    V[i + j * ldv] = v;
  }
}

// drand48_r stream, reseeded per leaf, row-major fill (init_matrix_tasks.cc:
// 66-76): x = (seed << 16) | 0x330E; x' = (0x5DEECE66D x + 0xB) mod 2^48.
__global__ void drand48_kernel(const int2 *__restrict__ leaves, int nleaves, double *B,
                               long long ldb, int m, long seed) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nleaves) return;
  const int2 lf = leaves[q];
  unsigned long long x = ((unsigned long long)(unsigned int)seed << 16) | 0x330Eull;
  const unsigned long long a = 0x5DEECE66Dull, c = 0xBull, mask = (1ull << 48) - 1;
  for (int i = 0; i < lf.y; ++i)
    for (int j = 0; j < m; ++j) {
      x = (a * x + c) & mask;
      B[lf.x + i + (long long)j * ldb] = ldexp((double)x, -48);
    }
}

// Philox4x32-10 (Salmon et al., "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): 10 rounds of the 4x32 bijection with the published multipliers
// and Weyl key increments.
__device__ inline uint4 philox4x32_10(uint4 ctr, uint2 key) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
    const uint32_t hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += W0;
    key.y += W1;
  }
  return ctr;
}

__device__ inline double u53(uint32_t hi, uint32_t lo) {
  // (0, 1]: 53 random bits, never zero (safe for log)
  const unsigned long long v = ((unsigned long long)hi << 21) ^ (unsigned long long)lo;
  return (double)((v & ((1ull << 53) - 1)) + 1) * 0x1.0p-53;
}

// a(i, j) = scale * N(0,1) [+ add on the diagonal i == j - diag_off]
// for i < rows, j < cols; `stream_id` separates independent fills.
__global__ void gauss_fill_kernel(double *a, long long lda, long long rows, long long cols,
                                  unsigned long long seed, unsigned int stream_id, double scale,
                                  double diag_add, long long diag_row0) {
  const long long total = rows * cols;
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  for (long long e2 = blockIdx.x * (long long)blockDim.x + threadIdx.x; 2 * e2 < total;
       e2 += (long long)gridDim.x * blockDim.x) {
    const uint4 ctr = make_uint4((uint32_t)e2, (uint32_t)(e2 >> 32), stream_id, 0x5eedu);
    const uint4 rv = philox4x32_10(ctr, key);
    const double u1 = u53(rv.x, rv.y), u2 = u53(rv.z, rv.w);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    const double g[2] = {rad * cs, rad * sn};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long e = 2 * e2 + h;
      if (e >= total) break;
      const long long i = e % rows, j = e / rows;
      double v = scale * g[h];
      if (i - diag_row0 == j) v += diag_add;
      a[i + j * lda] = v;
    }
  }
}

__global__ void gauss_fill_batched_kernel(const FillTask *__restrict__ tasks,
                                          unsigned long long seed) {
  const FillTask tk = tasks[blockIdx.y];
  const long long rows = tk.rows, total = rows * tk.cols;
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  for (long long e2 = blockIdx.x * (long long)blockDim.x + threadIdx.x; 2 * e2 < total;
       e2 += (long long)gridDim.x * blockDim.x) {
    const uint4 ctr = make_uint4((uint32_t)e2, (uint32_t)(e2 >> 32), tk.stream_id, 0x5eedu);
    const uint4 rv = philox4x32_10(ctr, key);
    const double u1 = u53(rv.x, rv.y), u2 = u53(rv.z, rv.w);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    const double g[2] = {rad * cs, rad * sn};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long e = 2 * e2 + h;
      if (e >= total) break;
      const long long i = e % rows, j = e / rows;
      double v = tk.scale * g[h];
      if (i == j) v += tk.diag_add;
      tk.a[i + j * tk.lda] = v;
    }
  }
}

__global__ void scale_batched_kernel(const FillTask *__restrict__ tasks) {
  const FillTask tk = tasks[blockIdx.y];
  const long long rows = tk.rows, total = rows * tk.cols;
  const double f = *tk.factor;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % rows, j = e / rows;
    tk.a[i + j * tk.lda] *= f;
  }
}

}  // namespace

void launch_gauss_fill_batched(const FillTask *tasks, int ntasks, long long max_elems,
                               unsigned long long seed, cudaStream_t s) {
  if (ntasks <= 0 || max_elems <= 0) return;
  const long long b = std::min<long long>(cdiv<long long>((max_elems + 1) / 2, kThreads), 1024);
  dim3 grid((unsigned)b, ntasks);
  gauss_fill_batched_kernel<<<grid, kThreads, 0, s>>>(tasks, seed);
  HODLR_LAUNCH_CHECK();
}

void launch_scale_batched(const FillTask *tasks, int ntasks, long long max_elems, cudaStream_t s) {
  if (ntasks <= 0 || max_elems <= 0) return;
  const long long b = std::min<long long>(cdiv<long long>(max_elems, kThreads), 1024);
  dim3 grid((unsigned)b, ntasks);
  scale_batched_kernel<<<grid, kThreads, 0, s>>>(tasks);
  HODLR_LAUNCH_CHECK();
}

template <typename TS, typename TD>
void launch_convert2d(const TS *src, long long lds, TD *dst, long long ldd, long long rows,
                      long long cols, cudaStream_t s) {
  launch_ew_tile<TS, TD, false>(src, lds, dst, ldd, rows, cols, s);
}
template void launch_convert2d<double, float>(const double *, long long, float *, long long,
                                              long long, long long, cudaStream_t);
template void launch_convert2d<float, double>(const float *, long long, double *, long long,
                                              long long, long long, cudaStream_t);
template void launch_convert2d<double, double>(const double *, long long, double *, long long,
                                               long long, long long, cudaStream_t);

template <typename TS>
void launch_add2d(double *x, long long ldx, const TS *y, long long ldy, long long rows,
                  long long cols, cudaStream_t s) {
  launch_ew_tile<TS, double, true>(y, ldy, x, ldx, rows, cols, s);
}
template void launch_add2d<float>(double *, long long, const float *, long long, long long,
                                  long long, cudaStream_t);
template void launch_add2d<double>(double *, long long, const double *, long long, long long,
                                   long long, cudaStream_t);

void launch_colratio(const double *r, long long ldr, const double *b, long long ldb,
                     long long rows, int cols, double *part, double *out, cudaStream_t s) {
  if (cols <= 0) return;
  const int nq = (int)std::max<long long>(1, std::min<long long>(kRatioChunks, (rows + 4095) / 4096));
  colratio_part_kernel<<<dim3(cols, nq), 256, 0, s>>>(r, ldr, b, ldb, rows, part);
  HODLR_LAUNCH_CHECK();
  colratio_fin_kernel<<<(cols + 127) / 128, 128, 0, s>>>(part, nq, cols, out);
  HODLR_LAUNCH_CHECK();
}

template <typename TS, typename TD>
void launch_ew2d_batched(const Ew2DTask<TS, TD> *tasks, int ntasks, long long total_tiles,
                         bool add, cudaStream_t s) {
  if (ntasks <= 0 || total_tiles <= 0) return;
  const unsigned grid = (unsigned)std::min<long long>(total_tiles, 148LL * 8);
  if (add) ew2d_batched_kernel<TS, TD, true><<<grid, kThreads, 0, s>>>(tasks, ntasks, total_tiles);
  else ew2d_batched_kernel<TS, TD, false><<<grid, kThreads, 0, s>>>(tasks, ntasks, total_tiles);
  HODLR_LAUNCH_CHECK();
}
template void launch_ew2d_batched<double, float>(const Ew2DTask<double, float> *, int, long long,
                                                 bool, cudaStream_t);
template void launch_ew2d_batched<float, double>(const Ew2DTask<float, double> *, int, long long,
                                                 bool, cudaStream_t);

void launch_colratio_batched(const RatioTask *tasks, int ntasks, int max_cols, cudaStream_t s) {
  if (ntasks <= 0 || max_cols <= 0) return;
  colratio_batched_kernel<<<dim3(max_cols, ntasks), 1024, 0, s>>>(tasks);
  HODLR_LAUNCH_CHECK();
}

template <typename T>
void launch_sum_slots(const SumTask<T> *tasks, int ntasks, long long max_len, cudaStream_t s) {
  if (ntasks <= 0 || max_len <= 0) return;
  // grid.y is at most 65535: merged batches can hold more tasks than that
  // about 16 CTAs per SM in all (each thread takes several elements): a grid
  // of one CTA per 256 elements of every task was ~34 k short CTAs at
  // N = 262144, bound by how fast CTAs start
  const long long per_task = std::max<long long>(1, 2368 / std::max(1, ntasks));
  for (int t0 = 0; t0 < ntasks; t0 += 65535) {
    dim3 grid((unsigned)std::min<long long>(cdiv<long long>(max_len, kThreads),
                                            std::min<long long>(per_task, 4096)),
              std::min(65535, ntasks - t0));
    sum_slots_kernel<T><<<grid, kThreads, 0, s>>>(tasks + t0);
    HODLR_LAUNCH_CHECK();
  }
}
template void launch_sum_slots<double>(const SumTask<double> *, int, long long, cudaStream_t);
template void launch_sum_slots<float>(const SumTask<float> *, int, long long, cudaStream_t);

void launch_scale_cols(double *a, long long lda, long long rows, int cols, const double *s_dev,
                       cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  scale_cols_kernel<<<grid_for(rows * cols), kThreads, 0, s>>>(a, lda, rows, cols, s_dev);
  HODLR_LAUNCH_CHECK();
}

void launch_circulant_k(const int2 *leaves, int nleaves, int max_leaf, double *D,
                        long long ldd, int r, double diag, cudaStream_t s) {
  if (nleaves <= 0) return;
  dim3 grid(cdiv<long long>((long long)max_leaf * max_leaf, kThreads), nleaves);
  circulant_k_kernel<<<grid, kThreads, 0, s>>>(leaves, nleaves, D, ldd, r, diag);
  HODLR_LAUNCH_CHECK();
}

void launch_circulant_uv(double *U, long long ldu, double *V, long long ldv, long long N,
                         int vcols, int r, cudaStream_t s) {
  if (N <= 0 || vcols <= 0) return;
  circulant_uv_kernel<<<grid_for(N * vcols), kThreads, 0, s>>>(U, ldu, V, ldv, N, vcols, r);
  HODLR_LAUNCH_CHECK();
}

void launch_drand48(const int2 *leaves, int nleaves, double *B, long long ldb, int m,
                    long seed, cudaStream_t s) {
  if (nleaves <= 0) return;
  drand48_kernel<<<cdiv(nleaves, 128), 128, 0, s>>>(leaves, nleaves, B, ldb, m, seed);
  HODLR_LAUNCH_CHECK();
}

void launch_gauss_fill(double *a, long long lda, long long rows, long long cols,
                       unsigned long long seed, unsigned int stream_id, double scale,
                       double diag_add, long long diag_row0, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  gauss_fill_kernel<<<grid_for((rows * cols + 1) / 2), kThreads, 0, s>>>(
      a, lda, rows, cols, seed, stream_id, scale, diag_add, diag_row0);
  HODLR_LAUNCH_CHECK();
}

}  // namespace hodlr
