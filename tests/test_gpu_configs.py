"""Parity at the benchmark workloads' exact shapes.

Each workload's system (seeded Gaussian HODLR: leaf blocks G/sqrt(n) + 2I,
U/V rescaled to off-diagonal spectral norm 0.5, b ~ N(0, 1)) is solved on the
GPU and by the oracle's restated FP64 walk (fast_solver.cc:136-255):

* N = 4096, leaf 256, r = 30, 1 RHS (the reference's CPU-runnable case) and
  N = 65536, leaf 512, r = 50, 8 RHS: the plain FP64 path within 1e-12 of
  the oracle (the reference's Err formula, direct_solve.cc:216-225), both
  node forms; the mixed path to relres <= 1e-12 with forward error < 1e-11;
* the rank-100, 32-RHS shape of the N = 2^20 workload at N = 16384 (the full
  size needs tens of GB of host memory for the oracle): mixed and FP64 paths
  vs the oracle, so the r = 100 node solve runs in both.
The N = 2^18 metric workload is checked at full size by bench.py (forward
error of both GPU paths against the oracle's solve of the same system).
"""
import numpy as np
import pytest

from gpu_util import relerr

pytestmark = pytest.mark.gpu

WORKLOADS = {
    "n4096_leaf256_r30_m1": (4096, 1, 30, 256),
    "n65536_leaf512_r50_m8": (65536, 8, 50, 512),
    "n16384_leaf512_r100_m32": (16384, 32, 100, 512),
}


def _system(fs, oracle, N, m, r, t, seed):
    s = oracle.gaussian_system(N, m, r, t, seed=seed)
    h = fs.HodlrMatrix(m, N, r, t).create_tree()
    h.set_matrix(s.D, s.U, s.V)
    h.set_rhs(s.B)
    return s, h


@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_workload_fp64_and_mixed_vs_oracle(fs, oracle, cuda, name):
    N, m, r, t = WORKLOADS[name]
    s, h = _system(fs, oracle, N, m, r, t, seed=1245667)
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    Xo = Xo[:, :m]
    sol = fs.FastSolver()
    forms = [False, True] if 2 * r <= 144 else [False]
    for schur2 in forms:
        sol.bfs_solve(h, schur2=schur2)
        x = h.solution()
        assert oracle.rel_error(x, Xo) < 1e-12, (name, schur2)
        assert oracle.relres(s, x) < 1e-13
    it, rr = sol.solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10)
    assert rr <= 1e-12
    x = h.solution()
    assert oracle.relres(s, x) <= 2e-12      # the oracle's matvec agrees
    assert relerr(x, Xo) < 1e-11             # forward error vs the FP64 oracle
