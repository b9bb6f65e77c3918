"""Whole-solve parity: the GPU tree walk against the oracle and the golden KAT.

* the reference's known-answer test, generated on the device, against the
  committed dense solutions (tests/golden) and against the oracle;
* seeded Gaussian systems (balanced and unbalanced trees) against the
  oracle's fused FP64 solve, both node forms;
* the factor/solve split and the mixed-precision refined solve, whose
  relative residual must reach 1e-12;
* the FP64 HODLR matvec against the oracle's.
FP64 tolerance: 1e-12 relative (Frobenius), the reference's Err formula.
"""
import numpy as np
import pytest

from gpu_util import dev, host, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def gpu_system(fs, s):
    h = fs.HodlrMatrix(s.m, s.N, int(s.tree[1, 1]) if s.tree.shape[0] > 1 else 1,
                       _threshold_of(s))
    h.create_tree()
    h.set_matrix(s.D, s.U if s.U.shape[1] else None, s.V if s.V.shape[1] else None)
    h.set_rhs(s.B)
    return h


def _threshold_of(s):
    return s.threshold


def make_gauss(oracle, N, m, r, t, seed):
    s = oracle.gaussian_system(N, m, r, t, seed=seed)
    s.threshold = t
    return s


@pytest.mark.parametrize("name", ["kat_n480", "kat_n201", "kat_n1000"])
def test_kat_on_device(fs, oracle, golden, cuda, name):
    g = golden(name)
    N, m, r, t = (int(g[k]) for k in ("N", "nrhs", "rank", "threshold"))
    h = fs.HodlrMatrix(m, N, r, t).create_tree()
    h.init_rhs(int(g["seed"]))
    h.init_circulant_matrix(float(g["diag"]))
    s = oracle.kat_system(N=N, nrhs=m, rank=r, threshold=t, diag=float(g["diag"]),
                          seed=int(g["seed"]))
    D, U, V, B = h.get_matrix()
    np.testing.assert_array_equal(B, g["B"])
    np.testing.assert_array_equal(D, s.D)
    np.testing.assert_array_equal(U, s.U)
    np.testing.assert_array_equal(V, s.V)
    fs.FastSolver().bfs_solve(h)
    x = h.solution()
    assert oracle.rel_error(x, g["X"]) < TOL           # the reference's Err vs dense
    Xo, _ = oracle.bfs_solve(s)
    assert relerr(x, Xo[:, :m]) < TOL                  # vs the restated HODLR walk


CASES = [(4096, 1, 30, 256), (4096, 8, 16, 300), (3001, 5, 12, 200), (777, 2, 8, 100),
         (20000, 4, 24, 512), (8192, 16, 64, 512), (65537, 3, 20, 1000)]


@pytest.mark.parametrize("N,m,r,t", CASES)
@pytest.mark.parametrize("schur2", [False, True])
def test_fused_fp64_vs_oracle(fs, oracle, cuda, N, m, r, t, schur2):
    s = make_gauss(oracle, N, m, r, t, seed=N + m)
    h = gpu_system(fs, s)
    fs.FastSolver().bfs_solve(h, schur2=schur2)
    x = h.solution()
    Xo, _ = oracle.bfs_solve(s, nthreads=8, schur2=schur2)
    assert relerr(x, Xo[:, :m]) < TOL
    assert oracle.relres(s, x) < 1e-13


@pytest.mark.parametrize("N,m,r,t", [(4096, 4, 16, 256), (20000, 3, 24, 512)])
def test_factor_then_solve_new_rhs(fs, oracle, cuda, N, m, r, t):
    s = make_gauss(oracle, N, m, r, t, seed=11)
    h = gpu_system(fs, s)
    solver = fs.FastSolver()
    solver.factor(h, fs.PREC_FP64)
    B2 = np.asfortranarray(np.random.default_rng(5).standard_normal((N, m)))
    h.set_rhs(B2)
    solver.solve(h)
    s.B = B2
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(h.solution(), Xo[:, :m]) < TOL


@pytest.mark.parametrize("N,m,r,t", [(4096, 1, 30, 256), (20000, 4, 24, 512),
                                     (65536, 8, 50, 512), (3001, 5, 12, 200)])
def test_mixed_refined_reaches_1e12(fs, oracle, cuda, N, m, r, t):
    s = make_gauss(oracle, N, m, r, t, seed=3 * N)
    h = gpu_system(fs, s)
    it, rr = fs.FastSolver().solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10)
    assert rr <= 1e-12
    x = h.solution()
    assert oracle.relres(s, x) <= 2e-12   # the oracle's matvec agrees
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(x, Xo[:, :m]) < 1e-11   # forward error vs the FP64 oracle


def test_matvec_vs_oracle(fs, oracle, cuda):
    s = make_gauss(oracle, 9000, 6, 20, 300, seed=4)
    h = gpu_system(fs, s)
    import torch
    x = np.asfortranarray(np.random.default_rng(9).standard_normal((9000, 6)))
    y = torch.zeros((6, 9000), dtype=torch.float64, device="cuda").T
    h.matvec(dev(x), y)
    assert relerr(host(y), oracle.matvec(s, x)) < 1e-13


def test_gaussian_generator_distribution(fs, oracle, cuda):
    N, m, r, t = 4096, 2, 16, 256
    h = fs.HodlrMatrix(m, N, r, t).create_tree()
    h.init_gaussian(1234, 0.5)
    D, U, V, B = h.get_matrix()
    tree = h.tree_nodes()
    s = oracle.System(tree, D, U, V, B)
    A = s.dense()
    F = oracle.F
    for p in range(tree.shape[0]):
        if tree[p, F["is_leaf"]]:
            continue
        c0, c1 = tree[p, F["lchild"]], tree[p, F["rchild"]]
        rs0 = slice(tree[c0, 2], tree[c0, 2] + tree[c0, 0])
        rs1 = slice(tree[c1, 2], tree[c1, 2] + tree[c1, 0])
        assert abs(np.linalg.norm(A[rs0, rs1], 2) - 0.5) < 1e-6
    assert abs(B.mean()) < 0.05 and abs(B.std() - 1) < 0.05
    leaf = D[:256, :256]
    off = (leaf - 2 * np.eye(256)) * 16.0
    assert abs(off.std() - 1) < 0.02
    # and the generated system solves like any other
    fs.FastSolver().bfs_solve(h)
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(h.solution(), Xo[:, :m]) < TOL


def test_solve_before_factor_is_state_error(fs, cuda):
    h = fs.HodlrMatrix(1, 1000, 8, 100).create_tree()
    with pytest.raises(fs.HodlrError) as e:
        fs.FastSolver().solve(h)
    assert e.value.status == fs.ERR_STATE


def test_singular_leaf_reported(fs, oracle, cuda):
    s = make_gauss(oracle, 2000, 1, 8, 250, seed=1)
    s.D[300, :] = 0.0   # zero row in leaf 2 -> exact zero pivot
    h = gpu_system(fs, s)
    with pytest.raises(fs.HodlrError) as e:
        fs.FastSolver().bfs_solve(h)
    assert e.value.status > 0


def test_save_solution_reference_format(fs, cuda, tmp_path):
    h = fs.HodlrMatrix(2, 480, 30, 60, name=str(tmp_path / "global")).create_tree()
    h.init_rhs(1245667)
    h.init_circulant_matrix(1.0e4)
    fs.FastSolver().bfs_solve(h)
    h.save_solution()
    rows = open(h.file_soln).read().splitlines()
    assert len(rows) == 480
    vals = np.array([[float(v) for v in r.split("\t") if v] for r in rows])
    np.testing.assert_array_equal(vals, h.solution())


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_graph_replay_new_rhs(fs, oracle, cuda, precision):
    """On a side stream the refined solve is captured as CUDA graphs on its
    first call and replayed afterwards: a second right-hand side loaded into
    the same system must be solved as accurately as the first, and the fused
    FP64 solve replayed on a third one must match the oracle."""
    import torch
    N, m, r, t = 8192, 3, 20, 256
    s = make_gauss(oracle, N, m, r, t, seed=11)
    h = gpu_system(fs, s)
    prec = fs.PREC_MIXED if precision == "mixed" else fs.PREC_FP64
    st = torch.cuda.Stream()
    sol = fs.FastSolver()
    rng = np.random.default_rng(5)
    for trial in range(3):
        B = np.asfortranarray(rng.standard_normal((N, m)))
        h.set_rhs(B, stream=st)
        s.B = B
        it, rr = sol.solve_refined(h, prec, tol=1e-12, maxiter=10, stream=st)
        st.synchronize()
        assert rr <= 1e-12, (trial, rr)
        x = h.solution(stream=st)
        Xo, _ = oracle.bfs_solve(s, nthreads=8)
        assert relerr(x, Xo[:, :m]) < 1e-11
    for trial in range(2):
        B = np.asfortranarray(rng.standard_normal((N, m)))
        h.set_rhs(B, stream=st)
        s.B = B
        sol.bfs_solve(h, stream=st)
        st.synchronize()
        Xo, _ = oracle.bfs_solve(s, nthreads=8)
        assert relerr(h.solution(stream=st), Xo[:, :m]) < 1e-12


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_solve_refined_host_matches_device_path(fs, oracle, cuda, precision):
    """The host-to-host refined solve (inputs copied in, V's copy under the
    leaf factorization for the mixed path, the solution copied out) gives
    bit for bit the solution of the device-resident solve, from pinned
    tensors on a side stream and from pageable arrays on the legacy stream,
    and repeated calls replay it unchanged."""
    import torch
    N, m, r, t = 20000, 4, 40, 512
    s = make_gauss(oracle, N, m, r, t, seed=31)
    prec = fs.PREC_MIXED if precision == "mixed" else fs.PREC_FP64
    h = gpu_system(fs, s)
    it1, rr1 = fs.FastSolver().solve_refined(h, prec, tol=1e-12, maxiter=10)
    x1 = h.solution()
    assert rr1 <= 1e-12

    def pinned(a):  # column-major pinned CPU tensor
        return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).pin_memory().t()

    h2 = fs.HodlrMatrix(m, N, r, t).create_tree()
    st = torch.cuda.Stream()
    sol = fs.FastSolver()
    x2, it2, rr2 = sol.solve_refined_host(h2, pinned(s.D), pinned(s.U), pinned(s.V), pinned(s.B),
                                          precision=prec, stream=st)
    assert it2 == it1 and rr2 == rr1
    np.testing.assert_array_equal(x2, x1)
    for _ in range(2):
        x3, it3, _ = sol.solve_refined_host(h2, s.D, s.U, s.V, s.B, precision=prec)
        assert it3 == it1
        np.testing.assert_array_equal(x3, x1)
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(x1, Xo[:, :m]) < 1e-11
