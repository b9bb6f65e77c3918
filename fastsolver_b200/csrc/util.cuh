// util.cuh -- element-wise kernels and device generators (util.cu).
#pragma once
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace hodlr {

// dst[t][0:len) = sum over q < nslots of src[t][q * stride + 0:len)
template <typename T>
struct SumTask {
  T *dst;
  const T *src;
  long long len;
  long long stride;
  int nslots;
  int pad;
};

template <typename TS, typename TD>
void launch_convert2d(const TS *src, long long lds, TD *dst, long long ldd, long long rows,
                      long long cols, cudaStream_t s);
template <typename TS>
void launch_add2d(double *x, long long ldx, const TS *y, long long ldy, long long rows,
                  long long cols, cudaStream_t s);
// out[c] = ||r(:, c)|| / ||b(:, c)|| (||r(:, c)|| where b(:, c) = 0), c < cols:
// every column is cut into up to kRatioChunks row chunks whose sums of
// squares land in `part` (cols x kRatioChunks x 2 doubles of scratch) and are
// added in a fixed order (deterministic).
constexpr int kRatioChunks = 64;
void launch_colratio(const double *r, long long ldr, const double *b, long long ldb,
                     long long rows, int cols, double *part, double *out, cudaStream_t s);
template <typename T>
void launch_sum_slots(const SumTask<T> *tasks, int ntasks, long long max_len, cudaStream_t s);
void launch_scale_cols(double *a, long long lda, long long rows, int cols, const double *s_dev,
                       cudaStream_t s);

void launch_circulant_k(const int2 *leaves, int nleaves, int max_leaf, double *D,
                        long long ldd, int r, double diag, cudaStream_t s);
void launch_circulant_uv(double *U, long long ldu, double *V, long long ldv, long long N,
                         int vcols, int r, cudaStream_t s);
void launch_drand48(const int2 *leaves, int nleaves, double *B, long long ldb, int m,
                    long seed, cudaStream_t s);
void launch_gauss_fill(double *a, long long lda, long long rows, long long cols,
                       unsigned long long seed, unsigned int stream_id, double scale,
                       double diag_add, long long diag_row0, cudaStream_t s);

// One block of a batched fill / scale: a(i, j), i < rows, j < cols.
struct FillTask {
  double *a;
  long long lda;
  int rows, cols;
  unsigned int stream_id;
  int pad;
  double scale;     // fill: N(0,1) * scale; scale task: factor index below
  double diag_add;  // fill: added on i == j
  const double *factor;  // scale task: a *= *factor
};
void launch_gauss_fill_batched(const FillTask *tasks, int ntasks, long long max_elems,
                               unsigned long long seed, cudaStream_t s);
void launch_scale_batched(const FillTask *tasks, int ntasks, long long max_elems, cudaStream_t s);

// One block of a batched element-wise pass over column-major matrices:
// dst(i, j) = TD(src(i, j)), or dst(i, j) += TD(src(i, j)).  The pass is cut
// into tiles of kEwTileRows rows of one column; tile0 = tiles of the tasks
// before this one (set by ew2d_prefix).
template <typename TS, typename TD>
struct Ew2DTask {
  const TS *src;
  long long lds;
  TD *dst;
  long long ldd;
  long long rows;
  long long cols;
  long long tile0;
};
constexpr int kEwTileRows = 1024;
inline long long ew2d_tiles(long long rows, long long cols) {
  return cdiv<long long>(rows, kEwTileRows) * cols;
}
// Sets every task's tile0 and returns the total tile count.
template <typename TS, typename TD>
long long ew2d_prefix(std::vector<Ew2DTask<TS, TD>> &tasks) {
  long long t = 0;
  for (auto &k : tasks) {
    k.tile0 = t;
    t += ew2d_tiles(k.rows, k.cols);
  }
  return t;
}
template <typename TS, typename TD>
void launch_ew2d_batched(const Ew2DTask<TS, TD> *tasks, int ntasks, long long total_tiles,
                         bool add, cudaStream_t s);

// Per-column residual ratios of one system of a batch:
// out[c] = ||r(:, c)|| / ||b(:, c)||, c < cols.
struct RatioTask {
  const double *r;
  long long ldr;
  const double *b;
  long long ldb;
  long long rows;
  double *out;
  int cols;
  int pad;
};
void launch_colratio_batched(const RatioTask *tasks, int ntasks, int max_cols, cudaStream_t s);

}  // namespace hodlr
