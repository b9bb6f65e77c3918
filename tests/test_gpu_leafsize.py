"""leafSize > 1: Legion leaves holding several real leaves
(mark_legion_leaf, hodlr_matrix.cc:317-337).

* the drand48 right-hand side is reseeded per Legion leaf (init_rhs,
  hodlr_matrix.cc:175-209): bit-exact against the oracle's KAT generator;
* the FP64 fused solve takes the 2r x 2r leaf-internal form
  (solver_tasks.cc:452-549) for the nodes inside a Legion leaf and the r x r
  LUSolve form above: within 1e-12 of the oracle's walk with the same
  granularity and of the dense solve of the reference's known-answer test;
* the text files hold one block (with its seed line) per Legion leaf, and
  load back bit-exactly.
"""
import numpy as np
import pytest

from gpu_util import relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("leaf_size", [1, 2, 4, 3])
def test_kat_leaf_size(fs, oracle, cuda, leaf_size, tmp_path):
    N, m, r, t, diag, seed = 960, 2, 30, 60, 1.0e4, 1245667
    h = fs.HodlrMatrix(m, N, r, t, leaf_size=leaf_size,
                       name=str(tmp_path / "global")).create_tree()
    h.init_rhs(seed)
    h.init_circulant_matrix(diag)
    s = oracle.kat_system(N=N, nrhs=m, rank=r, threshold=t, diag=diag, seed=seed,
                          leaf_size=leaf_size)
    assert h.get_num_leaf() == len(oracle.legion_leaves(s.tree, leaf_size))
    np.testing.assert_array_equal(list(h.legion_leaves()), oracle.legion_leaves(s.tree, leaf_size))
    D, U, V, B = h.get_matrix()
    np.testing.assert_array_equal(B, s.B)
    np.testing.assert_array_equal(D, s.D)
    fs.FastSolver().bfs_solve(h)
    x = h.solution()
    Xo, _ = oracle.bfs_solve(s, leaf_size=leaf_size)
    assert relerr(x, Xo[:, :m]) < 1e-12
    Xd = oracle.dense_solve(s.dense(), s.B)
    assert oracle.rel_error(x, Xd) < 1e-12
    # text files: one seed line per Legion leaf in the RHS file
    h.save_rhs()
    lines = open(h.file_rhs).read().splitlines()
    assert len(lines) == N + h.get_num_leaf()
    assert lines[0] == str(seed)
    h2 = fs.HodlrMatrix(m, N, r, t, leaf_size=leaf_size).create_tree()
    assert h2.load_rhs(h.file_rhs) == seed
    np.testing.assert_array_equal(h2.get_matrix()[3], B)
    h.save_solution()
    Y, _ = fs.read_text(h.file_soln, N, m)
    np.testing.assert_array_equal(Y, x)


@pytest.mark.parametrize("N,m,r,t,ls", [(8192, 3, 24, 256, 4), (3001, 2, 12, 200, 2),
                                        (20000, 4, 32, 512, 8)])
def test_gaussian_leaf_size(fs, oracle, cuda, N, m, r, t, ls):
    s = oracle.gaussian_system(N, m, r, t, seed=N + ls)
    h = fs.HodlrMatrix(m, N, r, t, leaf_size=ls).create_tree()
    h.set_matrix(s.D, s.U, s.V)
    h.set_rhs(s.B)
    fs.FastSolver().bfs_solve(h)
    Xo, _ = oracle.bfs_solve(s, nthreads=8, leaf_size=ls)
    assert relerr(h.solution(), Xo[:, :m]) < 1e-12
    assert oracle.relres(s, h.solution()) < 1e-13
    # the mixed path is unaffected by the granularity and refines to 1e-12
    it, rr = fs.FastSolver().solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10)
    assert rr <= 1e-12


def test_leaf_size_limits(fs, cuda):
    from fastsolver_b200._lib import lib
    h = fs.HodlrMatrix(1, 4096, 80, 512).create_tree()
    assert lib.hodlr_set_leaf_size(h.handle, 2) == fs.ERR_UNSUPPORTED   # 2r > 144
    assert lib.hodlr_set_leaf_size(h.handle, 0) == -2
    assert lib.hodlr_set_leaf_size(h.handle, 1) == 0
