// noalloc.cu -- a GEMM-reduce entry point that allocates no device memory.
//
// hodlr_gemm_reduce splits the K = k rows of V^T U into chunks, writes one
// partial product per chunk to scratch memory it obtains with
// cudaMallocAsync, and sums the partials in a fixed order into W.  Some
// callers cannot allocate device memory at all: a task body running under a
// runtime that owns the GPU's memory (Legion/Realm reserves the framebuffer at
// start-up and hands tasks only the regions they map), or a service that
// pre-reserves all device memory in its own pool.  hodlr_gemm_reduce_noalloc
// computes the same result with its scratch in a fixed-size array in the
// library's own device image (kNoAllocScratchDoubles doubles, 8 MiB), which
// every GPU that loads the library holds until the process exits.
//
// The array's name is a host-side stand-in in host code, not a device
// address: host code obtains the address with cudaGetSymbolAddress, once per
// device, with that device current, at the first call on that device.  All
// calls share the array, so calls that overlap on the GPU (different streams
// without ordering, or different host threads) race on it; the array keeps
// the previous call's partial sums, and every partial slot a call reads is
// written by that same call first.
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace hodlr {

namespace {

constexpr long long kNoAllocScratchDoubles = 1LL << 20;  // 8 MiB
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_addr[kMaxDevices] = {nullptr};

constexpr int NT = 256, BM = 64, BN = 64, BK = 16;

// One chunk of rows per blockIdx.x: P_q = V[rows_q]^T U[rows_q, col_beg:+ncol]
// (r x ncol, ld r) into scratch slot q.  The chunk, the operands and the slot
// layout are kernel parameters; nothing is read from descriptor memory.
__global__ void __launch_bounds__(NT)
    noalloc_partial_kernel(const double *__restrict__ V, long long ldv,
                           const double *__restrict__ U, long long ldu, int k, int r, int ncol,
                           int chunk, double *__restrict__ scratch) {
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN + 1];
  const int q = blockIdx.x;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.z * BN;
  const int kb = q * chunk, ke = min(k, kb + chunk);
  const int tid = threadIdx.x;
  const int tr = tid & 15, tc = tid >> 4;  // 4 x 4 outputs per thread
  double acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += BK) {
    for (int e = tid; e < BK * BM; e += NT) {
      const int kk = e % BK, mm = e / BK;
      const int gk = k0 + kk, gm = m0 + mm;
      As[kk][mm] = (gk < ke && gm < r) ? V[gk + (long long)gm * ldv] : 0.0;
    }
    for (int e = tid; e < BK * BN; e += NT) {
      const int kk = e % BK, nn = e / BK;
      const int gk = k0 + kk, gn = n0 + nn;
      Bs[kk][nn] = (gk < ke && gn < ncol) ? U[gk + (long long)gn * ldu] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][tr * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tc * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
  double *P = scratch + (long long)q * r * ncol;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gm = m0 + tr * 4 + i, gn = n0 + tc * 4 + j;
      if (gm < r && gn < ncol) P[gm + (long long)gn * r] = acc[i][j];
    }
}

// W(i, j) += alpha * sum_{q < nchunks} P_q(i, j), q in increasing order.
__global__ void noalloc_sum_kernel(const double *__restrict__ scratch, int nchunks, int r,
                                   int ncol, double alpha, double *__restrict__ W,
                                   long long ldw) {
  const long long total = (long long)r * ncol;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < nchunks; ++q) s += scratch[e + (long long)q * total];
    const long long i = e % r, j = e / r;
    W[i + j * ldw] += alpha * s;
  }
}

// Device address of the scratch array on the current device (first call on
// a device looks it up and caches it).
int scratch_address(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return HODLR_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return HODLR_ERR_CUDA;
    }
    g_addr[dev] = static_cast<double *>(p);
  }
  *out = g_addr[dev];
  return 0;
}

}  // namespace

}  // namespace hodlr

using namespace hodlr;

extern "C" int hodlr_gemm_reduce_noalloc(double alpha, int k, int r, int ncol, const double *V,
                                         int ldv, const double *U, int ldu, int col_beg,
                                         double *W, int ldw, hodlr_stream_t stream) {
  if (k < 0) return -2;
  if (r < 0) return -3;
  if (ncol < 0) return -4;
  if (!V && k > 0 && r > 0) return -5;
  if (ldv < (k > 1 ? k : 1)) return -6;
  if (!U && k > 0 && ncol > 0) return -7;
  if (ldu < (k > 1 ? k : 1)) return -8;
  if (col_beg < 0) return -9;
  if (!W && r > 0 && ncol > 0) return -10;
  if (ldw < (r > 1 ? r : 1)) return -11;
  if (r == 0 || ncol == 0) return 0;
  const long long slot = (long long)r * ncol;
  if (slot > kNoAllocScratchDoubles) return HODLR_ERR_UNSUPPORTED;  // r * ncol > 2^20
  if (k == 0) return 0;
  // as many row chunks as fit in the scratch, at least 1024 rows each
  long long nch = (k + 1023) / 1024;
  nch = std::min(nch, kNoAllocScratchDoubles / slot);
  if (nch < 1) nch = 1;
  const int chunk = (int)((k + nch - 1) / nch);
  const int nchunks = (k + chunk - 1) / chunk;
  double *scratch = nullptr;
  if (int e = scratch_address(&scratch)) return e;
  cudaStream_t s = as_stream(stream);
  dim3 grid(nchunks, (r + BM - 1) / BM, (ncol + BN - 1) / BN);
  noalloc_partial_kernel<<<grid, NT, 0, s>>>(V, ldv, U + (long long)col_beg * ldu, ldu, k, r, ncol,
                                             chunk, scratch);
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return HODLR_ERR_CUDA;
  const int sblocks = (int)std::min<long long>((slot + 255) / 256, 148 * 8);
  noalloc_sum_kernel<<<sblocks, 256, 0, s>>>(scratch, nchunks, r, ncol, alpha, W, ldw);
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return HODLR_ERR_CUDA;
  return 0;
}
