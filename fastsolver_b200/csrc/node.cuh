// node.cuh -- launchers of the capacitance (node) kernels (node.cu).
#pragma once
#include "common.cuh"

namespace hodlr {

// Largest capacitance system kept in shared memory (s = r or 2r).
constexpr int kMaxNodeS = 144;

size_t node_factor_smem(int max_s);
size_t node_apply_smem(int max_s, int max_rs, int form);

// One CTA per node: V^T u sums, S formation and LU (writes S_lu, S_piv, VTu*).
template <typename TW, typename TE>
void launch_node_factor(const NodeTask<TW, TE> *tasks, int count, int max_s, int form,
                        int *info, cudaStream_t s);

// eta0 / eta1 for every node, in chunks of columns of the d part.
template <typename TW, typename TE>
void launch_node_apply(const NodeTask<TW, TE> *tasks, int count, int max_s, int max_rs,
                       int max_c, int form, cudaStream_t s);

}  // namespace hodlr
