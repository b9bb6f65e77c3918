// gemm_simt.cuh -- launcher of the batched multi-segment SIMT GEMM.
#pragma once
#include "common.cuh"

namespace hodlr {

// Every item of `items` (device array) computes C = beta Cin + alpha sum op(A)B
// over its segments in `segs` (device array).  max_m / max_n bound the items'
// M / N (grid size).  trans selects op(A) = A^T (reduce) or A (broadcast).
template <typename TA, typename TC, typename TACC>
void launch_gemm_items(const GemmItem<TA, TC> *items, const GemmSeg<TA> *segs, int nitems,
                       int max_m, int max_n, bool trans, TACC alpha, TACC beta,
                       cudaStream_t s);

}  // namespace hodlr
