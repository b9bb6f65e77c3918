"""The allocation-free GEMM reduce, checked against the regular one.

hodlr_gemm_reduce_noalloc exists for callers that cannot allocate device
memory (a task body under a runtime that owns the GPU's memory, a service
with all device memory pre-reserved).  It keeps its split-K partial sums in a
fixed array in the library's device image instead of cudaMallocAsync'd
scratch.  Two calls in a row, with different shapes, must each match
hodlr_gemm_reduce on the same inputs and the oracle's reduce
(W += alpha V^T U[:, col_beg:col_beg+ncol], gemm.cc:376) to 1e-12 relative:
the second call also shows that the partial sums the first call left in the
shared array do not leak into its result.  This file is collected last.
"""
import numpy as np
import pytest

from gpu_util import dev, host, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _reduce(lib_fn, alpha, V, U, col_beg, ncol, W):
    import torch
    from fastsolver_b200._lib import lib
    k, r = V.shape
    st = getattr(lib, lib_fn)(float(alpha), k, r, ncol, V.data_ptr(), V.stride(1), U.data_ptr(),
                              U.stride(1), col_beg, W.data_ptr(), W.stride(1), None)
    torch.cuda.synchronize()
    return st


@pytest.mark.parametrize("calls", [[(131072, 64, 80, 16), (3000, 30, 92, 2)]])
def test_noalloc_reduce_matches_reduce(fs, oracle, cuda, calls):
    rng = np.random.default_rng(2024)
    for (k, r, ncol, col_beg) in calls:
        V = rng.standard_normal((k, r))
        U = rng.standard_normal((k, col_beg + ncol))
        W0 = rng.standard_normal((r, ncol))
        Vg, Ug = dev(V, k + 1), dev(U, k + 3)
        Wa, Wb = dev(W0, r + 2), dev(W0, r)
        assert _reduce("hodlr_gemm_reduce_noalloc", 0.5, Vg, Ug, col_beg, ncol, Wa) == 0
        assert _reduce("hodlr_gemm_reduce", 0.5, Vg, Ug, col_beg, ncol, Wb) == 0
        Wr = np.asfortranarray(W0.copy())
        Vf, Uf = np.asfortranarray(V), np.asfortranarray(U)
        oracle.lib().ref_gemm_reduce(0.5, k, r, ncol, oracle._p(Vf), k, oracle._p(Uf), k,
                                     col_beg, oracle._p(Wr), r)
        assert relerr(host(Wa), Wr) < TOL
        assert relerr(host(Wa), host(Wb)) < TOL


def test_noalloc_reduce_rejects_oversize(fs, cuda):
    from fastsolver_b200._lib import lib, ERR_UNSUPPORTED
    # r * ncol = 2048 * 1024 > 2^20 doubles of scratch: rejected before any
    # launch; k = 0 makes null V and U valid, and W is a real buffer of that
    # size, so no pointer of the call is a stand-in
    import torch
    W = torch.zeros((1024, 2048), dtype=torch.float64, device="cuda").T
    st = lib.hodlr_gemm_reduce_noalloc(1.0, 0, 2048, 1024, None, 1, None, 1, 0, W.data_ptr(),
                                       2048, None)
    assert st == ERR_UNSUPPORTED
