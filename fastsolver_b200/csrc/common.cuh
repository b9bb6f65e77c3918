// common.cuh -- shared definitions of the B200 HODLR solver library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

#include "../../include/hodlr_gpu.h"

namespace hodlr {

// ---------------------------------------------------------------------------
// Launch accounting and error plumbing
// ---------------------------------------------------------------------------

void count_launch();  // one per kernel launch issued by the library

struct CudaError {
  cudaError_t err;
};

#define HODLR_CUDA_TRY(expr)                                            \
  do {                                                                  \
    cudaError_t _e = (expr);                                            \
    if (_e != cudaSuccess) {                                            \
      fprintf(stderr, "hodlr: CUDA error %s at %s:%d: %s\n",            \
              cudaGetErrorName(_e), __FILE__, __LINE__,                 \
              cudaGetErrorString(_e));                                  \
      throw ::hodlr::CudaError{_e};                                     \
    }                                                                   \
  } while (0)

#define HODLR_LAUNCH_CHECK()                                            \
  do {                                                                  \
    ::hodlr::count_launch();                                            \
    HODLR_CUDA_TRY(cudaGetLastError());                                 \
  } while (0)

inline cudaStream_t as_stream(hodlr_stream_t s) {
  return reinterpret_cast<cudaStream_t>(s);
}

// ---------------------------------------------------------------------------
// Scalar helpers
// ---------------------------------------------------------------------------

template <typename T>
__host__ __device__ inline T cdiv(T a, T b) {
  return (a + b - 1) / b;
}

// ---------------------------------------------------------------------------
// Task descriptors (device-resident arrays, one launch per level)
// ---------------------------------------------------------------------------

// Leaf LU + solve.  T is the factor precision.
template <typename T>
struct LeafTask {
  T *D;          // n x n, ldd (overwritten by the LU factors)
  T *X;          // n x nrhs, ldx (overwritten by the solution)
  int *ipiv;     // n, LAPACK 1-based pivots
  int *perm;     // n, final row order
  long long ldd;
  long long ldx;
  int n;
  int nrhs;      // columns solved by getrs (0..nrhs-1 of X)
  int info_slot; // index into the info array
  int pad;
};

// One operand pair of a GEMM item: op(A) (M x K) times B (K x N).
//   TRANS (reduce):        A is K x M column-major (lda), op(A) = A^T
//   not TRANS (broadcast): A is M x K column-major (lda)
template <typename TA>
struct GemmSeg {
  const TA *A;
  const TA *B;  // K x N, ldb
  long long lda;
  long long ldb;
  int K;
  int pad;
};

// C (M x N) = beta * Cin + alpha * sum_s op(A_s) B_s over segments
// [seg_begin, seg_begin + seg_count).  Cin may alias C (in-place update) or
// be null (beta ignored).  Used for the reduce (one segment: V^T X over a row
// chunk, into a partial-sum slot), the broadcast (X -= U eta in place) and the
// matvec (r = b - D x - sum_d U_d t_d).
template <typename TA, typename TC>
struct GemmItem {
  TC *C;
  const TC *Cin;
  long long ldc;
  long long ldcin;
  int M, N;
  int seg_begin, seg_count;
};

// Capacitance (node) solve of one internal node with children b0, b1.  The
// reduce leaves, for child 0, `np0` partial sums (stride w0_stride apart) of
// V0^T d0 (r1 x c, at W0d, ld ldw0d) and of V0^T u0 (r1 x r0, at W0u, ld
// ldw0u); likewise for child 1.  The node kernels sum the partials in a fixed
// order.  `form` (a launch argument) 0 is LUSolveTask's r x r reduced system
// (solver_tasks.cc:139-305), 1 the 2r x 2r permuted Schur system of the
// leaf-internal branch (solver_tasks.cc:483-535).
template <typename TW, typename TE>
struct NodeTask {
  const TW *W0d, *W0u, *W1d, *W1u;
  long long w0_stride, w1_stride;
  long long ldw0d, ldw0u, ldw1d, ldw1u;
  TE *eta0;           // r0 x c out, ld ld_eta0: broadcast into child 0
  TE *eta1;           // r1 x c out, ld ld_eta1: broadcast into child 1
  long long ld_eta0, ld_eta1;
  double *S_lu;       // s x s: S before factoring (form 0), then its LU
  int *S_piv;         // s, 0-based pivot rows
  double *S_inv;      // s x s: S^{-1} from the LU factors
  double *VTu0;       // r1 x r0: V0^T u0 (factor writes, apply reads)
  double *VTu1;       // r0 x r1: V1^T u1
  int np0, np1;
  int r0, r1, c;
  int info_slot;
};

}  // namespace hodlr
