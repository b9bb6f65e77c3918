// tc_gemm.cuh -- split-BF16 tensor-core GEMM engine (tc_gemm.cu).
#pragma once
#include "common.cuh"

namespace hodlr {

// Same item semantics as launch_gemm_items (C = beta Cin + alpha sum op(A) B)
// for FP32 operands, computed on tcgen05 tensor cores as three BF16 products
// (hi*hi + hi*lo + lo*hi) accumulated in FP32.
template <typename TC>
void launch_tc_gemm(const GemmItem<float, TC> *items, const GemmSeg<float> *segs, int nitems,
                    int max_m, int max_n, bool trans, float alpha, float beta, cudaStream_t s);

// Device error flag raised by a tensor-core kernel whose bounded wait gave up
// (1), 0 if clear, -1 if it could not be read.
int tc_error_flag(bool reset);

// Test hook of the timeout path: every bounded wait of the engine gives up
// after `polls` tries (<= 0: the default, 2^22), and with skip_one_commit the
// next engine launch leaves out one completion signal, so one of its waits
// runs out; the kernel then raises the error flag, frees its tensor memory
// and returns.  Synchronous.
void tc_set_wait_hook(long long polls, int skip_one_commit);

}  // namespace hodlr
