"""The CPU oracle, pinned against the reference's known-answer test.

The reference has no golden vectors; its only results check is the dense
dgesv comparison of test/single_launch.cc:70-75 (direct_solve.cc:129-231).
tests/golden/ holds that dense side computed independently of the oracle
(numpy only, tests/golden/make_golden.py); these tests require the oracle's
restated HODLR solve to reproduce it.
"""
import ctypes

import numpy as np
import pytest


def _sys_from_golden(oracle, g):
    return oracle.kat_system(N=int(g["N"]), nrhs=int(g["nrhs"]), rank=int(g["rank"]),
                             threshold=int(g["threshold"]), diag=float(g["diag"]),
                             seed=int(g["seed"]))


@pytest.mark.parametrize("name", ["kat_n480", "kat_n201", "kat_n1000"])
def test_kat_rhs_is_golden(oracle, golden, name):
    g = golden(name)
    s = _sys_from_golden(oracle, g)
    np.testing.assert_array_equal(s.B, g["B"])


@pytest.mark.parametrize("name", ["kat_n480", "kat_n201", "kat_n1000"])
@pytest.mark.parametrize("schur2", [False, True])
def test_kat_solve_matches_golden(oracle, golden, name, schur2):
    g = golden(name)
    s = _sys_from_golden(oracle, g)
    X, _ = oracle.bfs_solve(s, schur2=schur2)
    err = oracle.rel_error(X[:, : s.m], g["X"])  # the reference's "Err:" formula
    assert err < 1e-12, err


def test_kat_dense_assembly_matches_formula(oracle, golden):
    g = golden("kat_n480")
    s = _sys_from_golden(oracle, g)
    A = s.dense()
    i = np.arange(s.N)[:, None]
    U = ((i + np.arange(30)[None, :]) % 30).astype(float)
    np.testing.assert_array_equal(A, 1.0e4 * np.eye(s.N) + U @ U.T)


def test_drand48_matches_glibc(oracle):
    libc = ctypes.CDLL("libc.so.6")

    class Drand48Data(ctypes.Structure):
        _fields_ = [("x", ctypes.c_ushort * 3), ("old_x", ctypes.c_ushort * 3),
                    ("c", ctypes.c_ushort), ("init", ctypes.c_ushort),
                    ("a", ctypes.c_ulonglong)]

    buf = Drand48Data()
    assert libc.srand48_r(ctypes.c_long(1245667), ctypes.byref(buf)) == 0
    ref = []
    v = ctypes.c_double()
    for _ in range(7 * 3):
        assert libc.drand48_r(ctypes.byref(buf), ctypes.byref(v)) == 0
        ref.append(v.value)
    out = oracle.fmat(7, 3)
    oracle.lib().ref_drand48_fill(1245667, 7, 3, oracle._p(out), 7)
    np.testing.assert_array_equal(out.reshape(-1), np.array(ref).reshape(7, 3).reshape(-1))


@pytest.mark.parametrize("N,m,r,t", [(4096, 1, 30, 256), (3001, 5, 12, 200), (777, 2, 8, 100)])
def test_gaussian_oracle_vs_dense(oracle, N, m, r, t):
    s = oracle.gaussian_system(N, m, r, t, seed=N)
    X, _ = oracle.bfs_solve(s, nthreads=4)
    xd = oracle.dense_solve(s.dense(), s.B)
    assert oracle.rel_error(X[:, :m], xd) < 1e-12
    assert oracle.relres(s, X[:, :m]) < 1e-13


def test_gaussian_offdiag_norm(oracle):
    s = oracle.gaussian_system(2048, 1, 16, 256, seed=3)
    A = s.dense()
    t, F = s.tree, oracle.F
    for p in range(t.shape[0]):
        if t[p, F["is_leaf"]]:
            continue
        c0, c1 = t[p, F["lchild"]], t[p, F["rchild"]]
        r0 = slice(t[c0, F["row_beg"]], t[c0, F["row_beg"]] + t[c0, F["nrow"]])
        r1 = slice(t[c1, F["row_beg"]], t[c1, F["row_beg"]] + t[c1, F["nrow"]])
        assert abs(np.linalg.norm(A[r0, r1], 2) - 0.5) < 1e-10
        assert abs(np.linalg.norm(A[r1, r0], 2) - 0.5) < 1e-10


def test_matvec_vs_dense(oracle):
    s = oracle.gaussian_system(1500, 3, 10, 100, seed=5)
    x = np.asfortranarray(np.random.default_rng(0).standard_normal((1500, 3)))
    np.testing.assert_allclose(oracle.matvec(s, x), s.dense() @ x, rtol=0, atol=1e-12)


def test_task_bodies_match_numpy(oracle):
    rng = np.random.default_rng(1)
    L = oracle.lib()
    # leaf solve
    n, c = 37, 11
    D = np.asfortranarray(rng.standard_normal((n, n)) + 3 * np.eye(n))
    X = np.asfortranarray(rng.standard_normal((n, c)))
    x = np.linalg.solve(D, X)
    Dc, Xc = D.copy(order="F"), X.copy(order="F")
    assert L.ref_leaf_solve(n, c, oracle._p(Dc), n, oracle._p(Xc), n, None) == 0
    np.testing.assert_allclose(Xc, x, rtol=1e-12, atol=1e-12)
    # node solve, both forms against the block system they restate
    r, cc = 6, 4
    V0Tu0 = np.asfortranarray(0.1 * rng.standard_normal((r, r)))
    V1Tu1 = np.asfortranarray(0.1 * rng.standard_normal((r, r)))
    V0Td0 = np.asfortranarray(rng.standard_normal((r, cc)))
    V1Td1 = np.asfortranarray(rng.standard_normal((r, cc)))
    S = np.block([[V0Tu0, np.eye(r)], [np.eye(r), V1Tu1]])
    sol = np.linalg.solve(S, np.vstack([V0Td0, V1Td1]))
    a, b = V0Td0.copy(order="F"), V1Td1.copy(order="F")
    assert L.ref_lu_node_solve(r, r, cc, oracle._p(V0Tu0), r, oracle._p(V1Tu1), r,
                               oracle._p(a), r, oracle._p(b), r) == 0
    np.testing.assert_allclose(b, sol[:r], rtol=1e-12, atol=1e-12)  # eta0 -> V1Td1
    np.testing.assert_allclose(a, sol[r:], rtol=1e-12, atol=1e-12)  # eta1 -> V0Td0
    a, b = V0Td0.copy(order="F"), V1Td1.copy(order="F")
    assert L.ref_schur2_solve(r, r, cc, oracle._p(V0Tu0), r, oracle._p(V1Tu1), r,
                              oracle._p(a), r, oracle._p(b), r) == 0
    np.testing.assert_allclose(a, sol[:r], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(b, sol[r:], rtol=1e-12, atol=1e-12)


def test_singular_leaf_reports_info(oracle):
    n = 8
    D = np.asfortranarray(np.eye(n))
    D[3, 3] = 0.0
    X = np.asfortranarray(np.ones((n, 1)))
    info = oracle.lib().ref_leaf_solve(n, 1, oracle._p(D), n, oracle._p(X), n, None)
    assert info == 4


def test_tree_layout(oracle):
    t = oracle.build_tree(262144, 16, 64, 512)
    F = oracle.F
    leaves = oracle.leaves(t)
    assert len(leaves) == 512
    assert all(t[i, F["nrow"]] == 512 and t[i, F["depth"]] == 9 for i in leaves)
    assert oracle.total_cols(t) == 16 + 64 * 9
    for i in range(1, t.shape[0]):
        p = t[i, F["parent"]]
        assert t[i, F["col_beg"]] == t[p, F["col_beg"]] + t[p, F["ncol"]]
