// leaf.cuh -- launchers of the batched leaf LU / solve kernels (leaf.cu).
#pragma once
#include "common.cuh"

namespace hodlr {

// LU with partial pivoting of every task's D (one CTA per leaf).  `tasks` is a
// device array of `count` tasks, or nullptr to use `single` (count must be 1).
template <typename T>
void launch_getrf(const LeafTask<T> *tasks, const LeafTask<T> &single, int count, int max_n,
                  int *info, cudaStream_t s);

// X <- (P L U)^{-1} X on columns [0, nrhs) of every task.
template <typename T>
void launch_getrs(const LeafTask<T> *tasks, const LeafTask<T> &single, int count, int max_n,
                  int max_nrhs, cudaStream_t s);

}  // namespace hodlr
