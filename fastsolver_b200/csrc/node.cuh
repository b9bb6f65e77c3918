// node.cuh -- launcher of the capacitance (node) factorization (node.cu).
#pragma once
#include "common.cuh"

namespace hodlr {

// Largest capacitance system kept in shared memory (s = r or 2r).
constexpr int kMaxNodeS = 144;

__host__ __device__ size_t node_factor_words(int max_s);
size_t node_factor_smem(int max_s);
// whether form-0 node factorization of nodes up to (max_s, max_r) stages
// V0Tu0, V1Tu1 in shared memory; then it also forms S = I - V1Tu1 V0Tu0
// itself (no separate product launch)
bool node_factor_stages(int max_s, int max_r);

// One CTA per node: S^{-1} (Gauss-Jordan, partial pivoting) and the node's
// solve matrix M; info[task.info_slot] = 0 or the first zero pivot (1-based).
template <typename TW, typename TE>
void launch_node_factor(const NodeTask<TW, TE> *tasks, int count, int max_s, int max_r, int form,
                        int *info, cudaStream_t s);

}  // namespace hodlr
