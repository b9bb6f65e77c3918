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
void add_launches(long long n);  // launches replayed by a CUDA graph
long long launch_total();

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

// Raises `func`'s dynamic shared-memory limit on the current device to at
// least `bytes` and never lowers it.  The limit is a property of the
// function, not of a launch or of a captured graph node: lowering it for a
// small launch would make an earlier-captured node that needs more fail at
// replay, so every launch site goes through this one monotonic setter.
void raise_smem_limit(const void *func, size_t bytes);

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
// One node of a level's capacitance factorization.  With the children's
// reduce results W0 = V0^T [d0 | u0] and W1 = V1^T [d1 | u1], the factor
// kernel writes the node's solve matrix M ((r0 + r1) x (r1 + r0), ld r0 + r1)
// such that [eta0; eta1] = M [V0Td0; V1Td1].
template <typename TW, typename TE>
struct NodeTask {
  const TW *W0u;      // V0^T u0: r1 x r0, ld ldw0u
  const TW *W1u;      // V1^T u1: r0 x r1, ld ldw1u
  long long ldw0u, ldw1u;
  const double *S;    // form 0: S = I - V1Tu1 V0Tu0 (r0 x r0, ld r0), FP64
  double *F;          // form 0: r1 x r0 FP64 work (-V0Tu0 S^{-1})
  TE *M;              // out: (r0 + r1)^2, ld r0 + r1
  int r0, r1;
  int info_slot;
  int pad;
};

}  // namespace hodlr
