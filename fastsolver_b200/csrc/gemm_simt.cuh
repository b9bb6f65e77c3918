// gemm_simt.cuh -- launcher of the batched multi-segment SIMT GEMM.
#pragma once
#include "common.cuh"

namespace hodlr {

// True unless the environment sets HODLR_TC=0 (FP32 GEMMs on the SIMT pipe).
bool tc_enabled();

// Every item of `items` (device array) computes C = beta Cin + alpha sum op(A)B
// over its segments in `segs` (device array).  max_m / max_n bound the items'
// M / N (grid size).  trans selects op(A) = A^T (reduce) or A (broadcast).
// FP32 items wider than 32 columns go to the tensor-core engine when
// allow_tc and tc_enabled().
template <typename TA, typename TC, typename TACC>
void launch_gemm_items(const GemmItem<TA, TC> *items, const GemmSeg<TA> *segs, int nitems,
                       int max_m, int max_n, bool trans, TACC alpha, TACC beta,
                       cudaStream_t s, bool allow_tc = true);

}  // namespace hodlr
