// node.cu -- capacitance (node) solves, FP64, batched over a tree level.
//
// GPU restatement of LUSolveTask::cpu_task (src/solver/solver_tasks.cc:
// 139-305) and of the 2r x 2r Schur system of serial_leaf_solve's internal
// branch (solver_tasks.cc:483-535).  Split in two kernels:
//
//   node_factor_kernel  one CTA per node: sums the reduce's partial products
//                       of V0^T u0 and V1^T u1 in a fixed order (the
//                       REDOP_ADD sum of gemm.cc:74-133, deterministic), forms
//                       S = I - V1Tu1 V0Tu0 (form 0) or [[V0Tu0, I], [I, V1Tu1]]
//                       (form 1), and factors it with partial pivoting in
//                       shared memory.  Keeps S's LU, pivots and both V^T u
//                       blocks for later solves with the same factorization.
//   node_apply_kernel   grid (column chunk, node): sums the partials of
//                       V0^T d0 and V1^T d1 for its columns and produces
//                       eta0 / eta1 exactly as the reference's dgemm / dgesv
//                       sequence does (form 0: V1Td1 -= V1Tu1 V0Td0;
//                       eta0 = S^{-1} V1Td1; eta1 = V0Td0 - V0Tu0 eta0).
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
  __shared__ int s_info;

  // V0Tu0 (r1 x r0) and V1Tu1 (r0 x r1): fixed-order sums of the partials
  for (int e = tid; e < r1 * r0; e += kNodeThreads) {
    const int i = e % r1, j = e / r1;
    const TW *p = tk.W0u + i + (long long)j * tk.ldw0u;
    double acc = 0.0;
    for (int q = 0; q < tk.np0; ++q) acc += double(p[(long long)q * tk.w0_stride]);
    tk.VTu0[i + (long long)j * r1] = acc;
  }
  for (int e = tid; e < r0 * r1; e += kNodeThreads) {
    const int i = e % r0, j = e / r0;
    const TW *p = tk.W1u + i + (long long)j * tk.ldw1u;
    double acc = 0.0;
    for (int q = 0; q < tk.np1; ++q) acc += double(p[(long long)q * tk.w1_stride]);
    tk.VTu1[i + (long long)j * r0] = acc;
  }
  if (tid == 0) s_info = 0;
  __syncthreads();

  if (form == 0) {
    // S = I - V1Tu1 * V0Tu0  (r0 x r0), k over r1
    for (int e = tid; e < r0 * r0; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      double acc = (i == j) ? 1.0 : 0.0;
      for (int k = 0; k < r1; ++k)
        acc -= tk.VTu1[i + (long long)k * r0] * tk.VTu0[k + (long long)j * r1];
      S[i + (size_t)j * s] = acc;
    }
  } else {
    for (int e = tid; e < s * s; e += kNodeThreads) S[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < s; i += kNodeThreads) S[(r1 + i) % s + (size_t)i * s] = 1.0;
    for (int e = tid; e < r1 * r0; e += kNodeThreads) {
      const int i = e % r1, j = e / r1;
      S[i + (size_t)j * s] = tk.VTu0[i + (long long)j * r1];
    }
    for (int e = tid; e < r0 * r1; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      S[(r1 + i) + (size_t)(r0 + j) * s] = tk.VTu1[i + (long long)j * r0];
    }
  }
  __syncthreads();

  // unblocked LU with partial pivoting; warp 0 picks and swaps the pivot row
  for (int j = 0; j < s; ++j) {
    if (warp == 0) {
      double best = -1.0;
      int bi = s;
      for (int i = j + lane; i < s; i += 32) {
        double a = fabs(S[i + (size_t)j * s]);
        if (a > best) { best = a; bi = i; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double ob = __shfl_down_sync(0xffffffffu, best, off);
        int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      bi = __shfl_sync(0xffffffffu, bi, 0);
      if (bi >= s) bi = j;
      if (bi != j)
        for (int c = lane; c < s; c += 32) {
          double t = S[j + (size_t)c * s];
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
      // one thread per row below the pivot (s <= kMaxNodeS <= kNodeThreads)
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
  if (tid == 0 && info) info[tk.info_slot] = s_info;
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
  const int rs = r0 + r1;                              // column stride of R
  double *S = reinterpret_cast<double *>(smem_raw);    // s x s
  double *R = S + (size_t)s * s;                       // rs x kApplyCols
  int *piv = reinterpret_cast<int *>(R + (size_t)rs * kApplyCols);
  // R rows [0, r1) = V0Td0, [r1, r1 + r0) = V1Td1 (form 1: the 2r RHS)
  for (int e = tid; e < s * s; e += kNodeThreads) S[e] = tk.S_lu[e];
  for (int i = tid; i < s; i += kNodeThreads) piv[i] = tk.S_piv[i];
  for (int e = tid; e < r1 * kApplyCols; e += kNodeThreads) {
    const int i = e % r1, j = e / r1;
    double acc = 0.0;
    if (j < cc) {
      const TW *p = tk.W0d + i + (long long)(cb + j) * tk.ldw0d;
      for (int q = 0; q < tk.np0; ++q) acc += double(p[(long long)q * tk.w0_stride]);
    }
    R[i + (size_t)j * rs] = acc;
  }
  for (int e = tid; e < r0 * kApplyCols; e += kNodeThreads) {
    const int i = e % r0, j = e / r0;
    double acc = 0.0;
    if (j < cc) {
      const TW *p = tk.W1d + i + (long long)(cb + j) * tk.ldw1d;
      for (int q = 0; q < tk.np1; ++q) acc += double(p[(long long)q * tk.w1_stride]);
    }
    R[r1 + i + (size_t)j * rs] = acc;
  }
  __syncthreads();

  double *y = (form == 0) ? R + r1 : R;  // the rows S acts on
  if (form == 0) {
    // V1Td1 -= V1Tu1 * V0Td0
    for (int e = tid; e < r0 * cc; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      double acc = R[r1 + i + (size_t)j * rs];
      for (int k = 0; k < r1; ++k) acc -= tk.VTu1[i + (long long)k * r0] * R[k + (size_t)j * rs];
      R[r1 + i + (size_t)j * rs] = acc;
    }
    __syncthreads();
  }
  // y <- S^{-1} y : interchanges, unit-lower forward, upper backward
  if (tid < cc) {
    double *col = y + (size_t)tid * rs;
    for (int j = 0; j < s; ++j) {
      const int p = piv[j];
      if (p != j) { double t = col[j]; col[j] = col[p]; col[p] = t; }
    }
    for (int i = 1; i < s; ++i) {
      double acc = col[i];
      for (int k = 0; k < i; ++k) acc -= S[i + (size_t)k * s] * col[k];
      col[i] = acc;
    }
    for (int i = s - 1; i >= 0; --i) {
      double acc = col[i];
      for (int k = i + 1; k < s; ++k) acc -= S[i + (size_t)k * s] * col[k];
      col[i] = acc / S[i + (size_t)i * s];
    }
  }
  __syncthreads();
  if (form == 0) {
    // eta1 = V0Td0 - V0Tu0 * eta0
    for (int e = tid; e < r1 * cc; e += kNodeThreads) {
      const int i = e % r1, j = e / r1;
      double acc = R[i + (size_t)j * rs];
      for (int k = 0; k < r0; ++k)
        acc -= tk.VTu0[i + (long long)k * r1] * R[r1 + k + (size_t)j * rs];
      R[i + (size_t)j * rs] = acc;
    }
    __syncthreads();
    for (int e = tid; e < r0 * cc; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      tk.eta0[i + (long long)(cb + j) * tk.ld_eta0] = TE(R[r1 + i + (size_t)j * rs]);
    }
    for (int e = tid; e < r1 * cc; e += kNodeThreads) {
      const int i = e % r1, j = e / r1;
      tk.eta1[i + (long long)(cb + j) * tk.ld_eta1] = TE(R[i + (size_t)j * rs]);
    }
  } else {
    for (int e = tid; e < r0 * cc; e += kNodeThreads) {
      const int i = e % r0, j = e / r0;
      tk.eta0[i + (long long)(cb + j) * tk.ld_eta0] = TE(R[i + (size_t)j * rs]);
    }
    for (int e = tid; e < r1 * cc; e += kNodeThreads) {
      const int i = e % r1, j = e / r1;
      tk.eta1[i + (long long)(cb + j) * tk.ld_eta1] = TE(R[r0 + i + (size_t)j * rs]);
    }
  }
}

}  // namespace

size_t node_factor_smem(int max_s) {
  return (size_t)max_s * max_s * sizeof(double) + (size_t)max_s * sizeof(int) + 16;
}
size_t node_apply_smem(int max_s, int max_rs) {
  return (size_t)max_s * max_s * sizeof(double) + (size_t)max_rs * kApplyCols * sizeof(double) +
         (size_t)max_s * sizeof(int) + 16;
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
  const size_t smem = node_apply_smem(max_s, max_rs);
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
template void launch_node_apply<double, double>(const NodeTask<double, double> *, int, int, int, int,
                                                int, cudaStream_t);
template void launch_node_apply<float, float>(const NodeTask<float, float> *, int, int, int, int,
                                                int, cudaStream_t);

}  // namespace hodlr
