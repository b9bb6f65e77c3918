// gemm_skinny.cuh -- batched GEMM items of at most 32 columns (gemm_skinny.cu).
#pragma once
#include "common.cuh"

namespace hodlr {

// C = beta Cin + alpha sum_s op(A_s) B_s for every item (N <= 32),
// op(A) = A^T when trans.
template <typename T>
void launch_skinny(const GemmItem<T, T> *items, const GemmSeg<T> *segs, int nitems, int max_m,
                   int max_n, bool trans, T alpha, T beta, cudaStream_t s);

}  // namespace hodlr
