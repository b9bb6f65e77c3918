// node.cu -- capacitance (node) solves, FP64, batched over a tree level.
//
// GPU restatement of LUSolveTask::cpu_task (src/solver/solver_tasks.cc:
// 139-305) and of the 2r x 2r Schur system of serial_leaf_solve's internal
// branch (solver_tasks.cc:483-535).  For a node with children b0, b1 and the
// summed reduce results W0 = [V0Td0 | V0Tu0], W1 = [V1Td1 | V1Tu1]:
//
//   node_factor_kernel  one CTA per node.  Form 0: S = I - V1Tu1 V0Tu0 has
//                       been written into S_lu by a batched GEMM launch; form
//                       1 assembles [[V0Tu0, I], [I, V1Tu1]] here.  Factors S
//                       with partial pivoting (LAPACK getrf semantics, lowest
//                       index on ties), stores the LU and pivots, then forms
//                       S^{-1} = U^{-1} L^{-1} P from the factors (in-place
//                       triangular inverses in shared memory) and keeps both
//                       V^T u blocks for later solves with the same factors.
//   node_apply_kernel   grid (column chunk, node).  Form 0, as the
//                       reference's dgemm / dgesv sequence:
//                         T    = V1Td1 - V1Tu1 V0Td0   (dgemm at 236)
//                         eta0 = S^{-1} T              (dgesv at 281)
//                         eta1 = V0Td0 - V0Tu0 eta0    (dgemm at 299)
//                       form 1: [eta0; eta1] = S^{-1} [V0Td0; V1Td1].
//                       The three products run from shared memory, so the
//                       kernel is fully parallel over columns and nodes.
#include "common.cuh"
#include "node.cuh"

namespace hodlr {

namespace {

constexpr int kNodeThreads = 256;
constexpr int kApplyCols = 32;

template <typename TW, typename TE>
__global__ void __launch_bounds__(kNodeThreads)
    node_factor_kernel(const NodeTask<TW, TE> *tasks, int form, int *info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const NodeTask<TW, TE> tk = tasks[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = tk.r0, r1 = tk.r1;
  const int s = form == 0 ? r0 : r0 + r1;
  double *S = reinterpret_cast<double *>(smem_raw);  // s x s, column-major
  int *piv = reinterpret_cast<int *>(S + (size_t)s * s);
  int *perm = piv + s;
  __shared__ int s_info;

  // keep V0^T u0 (r1 x r0) and V1^T u1 (r0 x r1) for solves with these factors
  for (int e = tid; e < r1 * r0; e += kNodeThreads) {
    const int i = e % r1, j = e / r1;
    tk.VTu0[e] = double(tk.W0u[i + (long long)j * tk.ldw0u]);
  }
  for (int e = tid; e < r0 * r1; e += kNodeThreads) {
    const int i = e % r0, j = e / r0;
    tk.VTu1[e] = double(tk.W1u[i + (long long)j * tk.ldw1u]);
  }
  if (tid == 0) s_info = 0;
  if (form == 0) {
    for (int e = tid; e < s * s; e += kNodeThreads) S[e] = tk.S_lu[e];
  } else {
    for (int e = tid; e < s * s; e += kNodeThreads) S[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < s; i += kNodeThreads) S[(r1 + i) % s + (size_t)i * s] = 1.0;
    for (int e = tid; e < r1 * r0; e += kNodeThreads) {
      const int i = e % r1, j = e / r1;
      S[i + (size_t)j * s] = double(tk.W0u[i + (long long)j * tk.ldw0u]);
    }
    for (int e = tid; e < r0 * r1; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      S[(r1 + i) + (size_t)(r0 + j) * s] = double(tk.W1u[i + (long long)j * tk.ldw1u]);
    }
  }
  __syncthreads();

  // ---- LU with partial pivoting; warp 0 picks and swaps the pivot row
  for (int j = 0; j < s; ++j) {
    if (warp == 0) {
      double best = -1.0;
      int bi = s;
      for (int i = j + lane; i < s; i += 32) {
        const double a = fabs(S[i + (size_t)j * s]);
        if (a > best) { best = a; bi = i; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      bi = __shfl_sync(0xffffffffu, bi, 0);
      if (bi >= s) bi = j;
      if (bi != j)
        for (int c = lane; c < s; c += 32) {
          const double t = S[j + (size_t)c * s];
          S[j + (size_t)c * s] = S[bi + (size_t)c * s];
          S[bi + (size_t)c * s] = t;
        }
      if (lane == 0) {
        piv[j] = bi;
        if (S[j + (size_t)j * s] == 0.0 && s_info == 0) s_info = j + 1;
      }
    }
    __syncthreads();
    const double pv = S[j + (size_t)j * s];
    if (pv != 0.0) {
      const double rinv = 1.0 / pv;
      for (int row = j + 1 + tid; row < s; row += kNodeThreads) {
        const double l = S[row + (size_t)j * s] * rinv;
        for (int c = j + 1; c < s; ++c) S[row + (size_t)c * s] -= l * S[j + (size_t)c * s];
        S[row + (size_t)j * s] = l;
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < s * s; e += kNodeThreads) tk.S_lu[e] = S[e];
  for (int i = tid; i < s; i += kNodeThreads) tk.S_piv[i] = piv[i];
  if (tid == 0) {
    if (info) info[tk.info_slot] = s_info;
    for (int i = 0; i < s; ++i) perm[i] = i;
    for (int j = 0; j < s; ++j) {
      const int p = piv[j];
      if (p != j) { const int t = perm[j]; perm[j] = perm[p]; perm[p] = t; }
    }
  }
  __syncthreads();
  if (s_info != 0) return;  // singular: no inverse (uniform across the CTA)

  // ---- L^{-1} in place (unit lower), columns right to left
  for (int j = s - 2; j >= 0; --j) {
    double v = 0.0;
    const int i = j + 1 + tid;
    if (i < s) {
      v = S[i + (size_t)j * s];
      for (int k = j + 1; k < i; ++k) v += S[i + (size_t)k * s] * S[k + (size_t)j * s];
      v = -v;
    }
    __syncthreads();
    if (i < s) S[i + (size_t)j * s] = v;
    __syncthreads();
  }
  // ---- U^{-1} in place (upper), columns left to right
  for (int j = 0; j < s; ++j) {
    const double ujj = S[j + (size_t)j * s];
    double v = 0.0;
    const int i = tid;
    if (i < j) {
      for (int k = i; k < j; ++k) v += S[i + (size_t)k * s] * S[k + (size_t)j * s];
      v = -v / ujj;
    }
    __syncthreads();
    if (i < j) S[i + (size_t)j * s] = v;
    if (i == j) S[j + (size_t)j * s] = 1.0 / ujj;
    __syncthreads();
  }
  // ---- S^{-1}[:, perm[q]] = (U^{-1} L^{-1})[:, q]
  for (int e = tid; e < s * s; e += kNodeThreads) {
    const int i = e % s, q = e / s;
    double acc = 0.0;
    for (int k = max(i, q); k < s; ++k) {
      const double lk = (k == q) ? 1.0 : S[k + (size_t)q * s];
      acc += S[i + (size_t)k * s] * lk;
    }
    tk.S_inv[i + (size_t)perm[q] * s] = acc;
  }
}

// Y (M x cc, ld ldy) = Y0 (or 0) + alpha * A (M x K, ld M) * X (K x cc, ld
// ldx); all in shared memory, Y aliases neither A nor X.
__device__ inline void smem_gemm(double *Y, int ldy, const double *Y0, int ldy0, double alpha,
                                 const double *A, int M, int K, const double *X, int ldx, int cc) {
  for (int e = threadIdx.x; e < M * cc; e += kNodeThreads) {
    const int i = e % M, c = e / M;
    double acc = 0.0;
    const double *xc = X + (size_t)c * ldx;
#pragma unroll 4
    for (int k = 0; k < K; ++k) acc += A[i + (size_t)k * M] * xc[k];
    Y[i + (size_t)c * ldy] = (Y0 ? Y0[i + (size_t)c * ldy0] : 0.0) + alpha * acc;
  }
}

template <typename TE>
__device__ inline void store_eta(TE *eta, long long ld, int cb, const double *Y, int ldy, int M,
                                 int cc) {
  for (int e = threadIdx.x; e < M * cc; e += kNodeThreads) {
    const int i = e % M, c = e / M;
    eta[i + (long long)(cb + c) * ld] = TE(Y[i + (size_t)c * ldy]);
  }
}

template <typename TW, typename TE>
__global__ void __launch_bounds__(kNodeThreads)
    node_apply_kernel(const NodeTask<TW, TE> *tasks, int form) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const NodeTask<TW, TE> tk = tasks[blockIdx.y];
  const int cb = blockIdx.x * kApplyCols;
  if (cb >= tk.c) return;
  const int cc = min(kApplyCols, tk.c - cb);
  const int tid = threadIdx.x;
  const int r0 = tk.r0, r1 = tk.r1;
  const int s = form == 0 ? r0 : r0 + r1;
  const int rs = r0 + r1;
  double *A = reinterpret_cast<double *>(smem_raw);  // staged matrix, <= s x s
  double *R = A + (size_t)s * s;                     // rs x kApplyCols: [V0Td0; V1Td1]
  double *T = R + (size_t)rs * kApplyCols;           // form 0: max(r0, r1) x kApplyCols
  for (int e = tid; e < r1 * cc; e += kNodeThreads) {
    const int i = e % r1, j = e / r1;
    R[i + (size_t)j * rs] = double(tk.W0d[i + (long long)(cb + j) * tk.ldw0d]);
  }
  for (int e = tid; e < r0 * cc; e += kNodeThreads) {
    const int i = e % r0, j = e / r0;
    R[r1 + i + (size_t)j * rs] = double(tk.W1d[i + (long long)(cb + j) * tk.ldw1d]);
  }
  if (form == 0) {
    for (int e = tid; e < r0 * r1; e += kNodeThreads) A[e] = tk.VTu1[e];
    __syncthreads();
    // T = V1Td1 - V1Tu1 V0Td0
    smem_gemm(T, r0, R + r1, rs, -1.0, A, r0, r1, R, rs, cc);
    __syncthreads();
    for (int e = tid; e < r0 * r0; e += kNodeThreads) A[e] = tk.S_inv[e];
    __syncthreads();
    // eta0 = S^{-1} T into the V1Td1 rows of R
    smem_gemm(R + r1, rs, nullptr, 0, 1.0, A, r0, r0, T, r0, cc);
    __syncthreads();
    for (int e = tid; e < r1 * r0; e += kNodeThreads) A[e] = tk.VTu0[e];
    __syncthreads();
    // eta1 = V0Td0 - V0Tu0 eta0 into T
    smem_gemm(T, r1, R, rs, -1.0, A, r1, r0, R + r1, rs, cc);
    __syncthreads();
    store_eta(tk.eta0, tk.ld_eta0, cb, R + r1, rs, r0, cc);
    store_eta(tk.eta1, tk.ld_eta1, cb, T, r1, r1, cc);
  } else {
    for (int e = tid; e < s * s; e += kNodeThreads) A[e] = tk.S_inv[e];
    __syncthreads();
    // [eta0; eta1] = S^{-1} [V0Td0; V1Td1], straight to global
    for (int e = tid; e < s * cc; e += kNodeThreads) {
      const int i = e % s, c = e / s;
      double acc = 0.0;
      const double *xc = R + (size_t)c * rs;
#pragma unroll 4
      for (int k = 0; k < s; ++k) acc += A[i + (size_t)k * s] * xc[k];
      if (i < r0) tk.eta0[i + (long long)(cb + c) * tk.ld_eta0] = TE(acc);
      else tk.eta1[(i - r0) + (long long)(cb + c) * tk.ld_eta1] = TE(acc);
    }
  }
}

}  // namespace

size_t node_factor_smem(int max_s) {
  return (size_t)max_s * max_s * sizeof(double) + 2 * (size_t)max_s * sizeof(int) + 16;
}
size_t node_apply_smem(int max_s, int max_rs, int form) {
  // A (s x s) + R (rs x 32) + T (form 0 only, <= rs x 32)
  return (size_t)max_s * max_s * sizeof(double) + (size_t)max_rs * kApplyCols * sizeof(double) +
         (form == 0 ? (size_t)max_rs * kApplyCols * sizeof(double) : 0) + 16;
}

template <typename TW, typename TE>
void launch_node_factor(const NodeTask<TW, TE> *tasks, int count, int max_s, int form,
                        int *info, cudaStream_t s) {
  if (count <= 0) return;
  const size_t smem = node_factor_smem(max_s);
  HODLR_CUDA_TRY(cudaFuncSetAttribute(node_factor_kernel<TW, TE>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  node_factor_kernel<TW, TE><<<count, kNodeThreads, smem, s>>>(tasks, form, info);
  HODLR_LAUNCH_CHECK();
}

template <typename TW, typename TE>
void launch_node_apply(const NodeTask<TW, TE> *tasks, int count, int max_s, int max_rs,
                       int max_c, int form, cudaStream_t s) {
  if (count <= 0 || max_c <= 0) return;
  const size_t smem = node_apply_smem(max_s, max_rs, form);
  HODLR_CUDA_TRY(cudaFuncSetAttribute(node_apply_kernel<TW, TE>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(cdiv(max_c, kApplyCols), count);
  node_apply_kernel<TW, TE><<<grid, kNodeThreads, smem, s>>>(tasks, form);
  HODLR_LAUNCH_CHECK();
}

template void launch_node_factor<double, double>(const NodeTask<double, double> *, int, int,
                                                 int, int *, cudaStream_t);
template void launch_node_factor<float, float>(const NodeTask<float, float> *, int, int, int,
                                               int *, cudaStream_t);
template void launch_node_apply<double, double>(const NodeTask<double, double> *, int, int, int,
                                                int, int, cudaStream_t);
template void launch_node_apply<float, float>(const NodeTask<float, float> *, int, int, int, int,
                                              int, cudaStream_t);

}  // namespace hodlr
