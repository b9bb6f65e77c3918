// node.cuh -- launcher of the capacitance (node) factorization (node.cu).
#pragma once
#include "common.cuh"

namespace hodlr {

// Largest capacitance system kept in shared memory (s = r or 2r).
constexpr int kMaxNodeS = 144;

__host__ __device__ size_t node_factor_words(int max_s);
size_t node_factor_smem(int max_s);

// One CTA per node: S^{-1} (Gauss-Jordan, partial pivoting) and the node's
// solve matrix M; info[task.info_slot] = 0 or the first zero pivot (1-based).
template <typename TW, typename TE>
void launch_node_factor(const NodeTask<TW, TE> *tasks, int count, int max_s, int max_r, int form,
                        int *info, cudaStream_t s);

}  // namespace hodlr
