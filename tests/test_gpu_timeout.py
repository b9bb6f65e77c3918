"""The tensor-core engine's bounded waits, made to run out from the host.

hodlr_debug_tc_wait_hook shortens every mbarrier wait of the engine and asks
the next engine launch to leave out one tile's completion signal, so the
epilogue's wait for that tile runs out.  The kernel must then raise the
device error flag, wait (bounded) for its own tensor-core work, free its
tensor memory and return -- no trap, no fault, no hang -- and the calls that
synchronize must report HODLR_ERR_TIMEOUT.  The next call, with the hook
cleared, must succeed and be correct: the context and the tensor memory are
still usable.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POLLS = 1 << 18   # >= a few ms per wait: far above any healthy wait of these sizes


def _hook(polls, skip):
    from fastsolver_b200._lib import lib
    assert lib.hodlr_debug_tc_wait_hook(polls, skip) == 0


def _gemm(m, n, k, seed):
    import torch
    from fastsolver_b200._lib import lib
    g = torch.Generator(device="cpu").manual_seed(seed)
    A = torch.randn((m, k), generator=g, dtype=torch.float32)
    B = torch.randn((k, n), generator=g, dtype=torch.float32)
    Ad = A.t().contiguous().cuda().t()
    Bd = B.t().contiguous().cuda().t()
    Cd = torch.zeros((n, m), dtype=torch.float32, device="cuda").t()
    st = lib.hodlr_gemm_f32(0, m, n, k, 1.0, Ad.data_ptr(), Ad.stride(1), Bd.data_ptr(),
                            Bd.stride(1), 0.0, Cd.data_ptr(), Cd.stride(1), 1, None)
    ref = A.double() @ B.double()
    err = ((Cd.cpu().double() - ref).abs().max() / ref.abs().max()).item()
    return st, err


def test_gemm_timeout_reported_then_recovers(fs, cuda):
    from fastsolver_b200._lib import ERR_TIMEOUT
    try:
        _hook(POLLS, 1)
        st, _ = _gemm(256, 256, 64, 1)
        assert st == ERR_TIMEOUT
    finally:
        _hook(0, 0)
    st, err = _gemm(256, 256, 64, 2)
    assert st == 0 and err < 1e-4


def test_refined_solve_timeout_reported_then_recovers(fs, oracle, cuda):
    import torch
    from gpu_util import relerr
    N, m, r, t = 8192, 3, 20, 256
    s = oracle.gaussian_system(N, m, r, t, seed=21)
    h = fs.HodlrMatrix(m, N, r, t).create_tree()
    h.set_matrix(s.D, s.U, s.V)
    h.set_rhs(s.B)
    sol = fs.FastSolver()
    st = torch.cuda.Stream()
    # first solve captures the graphs; the failing one replays them
    it, rr = sol.solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10, stream=st)
    assert rr <= 1e-12
    try:
        _hook(POLLS, 1)
        with pytest.raises(fs.HodlrError) as e:
            sol.solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10, stream=st)
        assert e.value.status == fs.ERR_TIMEOUT
    finally:
        _hook(0, 0)
    it, rr = sol.solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10, stream=st)
    assert rr <= 1e-12
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(h.solution(stream=st), Xo[:, :m]) < 1e-11


def test_sweep_barrier_timeout_reported_then_recovers(fs, oracle, cuda):
    """The persistent sweep kernel's grid barrier: one CTA leaves before its
    first arrival, the others' bounded waits run out and the kernel ends; the
    refined solve reports HODLR_ERR_TIMEOUT and the next one is correct."""
    import torch
    from fastsolver_b200._lib import lib
    from gpu_util import relerr
    N, m, r, t = 8192, 3, 20, 256
    s = oracle.gaussian_system(N, m, r, t, seed=23)
    h = fs.HodlrMatrix(m, N, r, t).create_tree()
    h.set_matrix(s.D, s.U, s.V)
    h.set_rhs(s.B)
    sol = fs.FastSolver()
    st = torch.cuda.Stream()
    it, rr = sol.solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10, stream=st)
    assert rr <= 1e-12 and it >= 1     # at least one sweep: the kernel ran
    try:
        assert lib.hodlr_debug_sweep_barrier_hook(POLLS, 1) == 0
        with pytest.raises(fs.HodlrError) as e:
            sol.solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10, stream=st)
        assert e.value.status == fs.ERR_TIMEOUT
    finally:
        assert lib.hodlr_debug_sweep_barrier_hook(0, 0) == 0
    it, rr = sol.solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10, stream=st)
    assert rr <= 1e-12
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(h.solution(stream=st), Xo[:, :m]) < 1e-11
