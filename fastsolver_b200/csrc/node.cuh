// node.cuh -- launcher of the capacitance (node) factorization (node.cu).
#pragma once
#include <vector>

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
// g_alias: every node of the launch has r1 <= r0 + 1, so that the staged
// form-0 kernel may keep G0 = -S^{-1} V1Tu1 in the eliminated matrix's
// shared memory (less shared memory per CTA: two CTAs per SM for the FP32
// path at r = 64).
template <typename TW, typename TE>
void launch_node_factor(const NodeTask<TW, TE> *tasks, int count, int max_s, int max_r, int form,
                        int *info, cudaStream_t s, bool g_alias = false);

// whether G0 of every form-0 node in `tasks` (host copies) fits in the
// eliminated matrix's shared memory: r0 r1 <= r0 (r0 + 1)
template <typename TW, typename TE>
bool node_g_alias(const std::vector<NodeTask<TW, TE>> &tasks) {
  for (const auto &t : tasks)
    if (t.r1 > t.r0 + 1) return false;
  return true;
}

}  // namespace hodlr
