"""fastsolver_b200 -- HODLR direct solver for NVIDIA B200 (sm_100a).

A from-scratch GPU implementation of the hot path of Charles-Chao-Chen/
fastSolver: the leaf solve, GEMM reduce, capacitance (node) LU and GEMM
broadcast task bodies and the tree walk that drives them.  The native library
(libhodlr_b200.so: C++ host code + CUDA kernels behind the C ABI in
include/hodlr_gpu.h) does all the work; this package is its Python front end.
"""
from ._lib import (ERR_CUDA, ERR_IO, ERR_NOCONV, ERR_NOMEM, ERR_STATE, ERR_TIMEOUT,
                   ERR_UNSUPPORTED,
                   HODLR_OK, LIB_PATH, NODE_FIELDS, PREC_FP64, PREC_MIXED, HodlrError,
                   launch_count, reset_launch_count)
from .hodlr import (FastSolver, HodlrMatrix, SystemBatch, build_tree, gemm_broadcast,
                    gemm_reduce, leaf_solve, node_lu_solve, node_schur2_solve, read_text,
                    write_text)

__all__ = [
    "HodlrMatrix", "FastSolver", "SystemBatch", "build_tree", "leaf_solve", "gemm_reduce",
    "gemm_broadcast",
    "node_lu_solve", "node_schur2_solve", "PREC_FP64", "PREC_MIXED", "HodlrError",
    "launch_count", "reset_launch_count", "LIB_PATH", "NODE_FIELDS", "HODLR_OK", "ERR_CUDA",
    "ERR_NOMEM", "ERR_STATE", "ERR_NOCONV", "ERR_TIMEOUT", "ERR_UNSUPPORTED", "ERR_IO",
    "read_text", "write_text",
]
