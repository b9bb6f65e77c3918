// gemm_dmma.cuh -- batched FP64 GEMM items on the DMMA pipe (gemm_dmma.cu).
#pragma once
#include "common.cuh"

namespace hodlr {

// C = beta Cin + alpha sum_s op(A_s) B_s for every FP64 item, op(A) = A^T
// when trans; max_m / max_n bound the items' M / N (grid size).
void launch_dmma_tile(const GemmItem<double, double> *items, const GemmSeg<double> *segs,
                      int nitems, int max_m, int max_n, bool trans, double alpha, double beta,
                      cudaStream_t s);

}  // namespace hodlr
