"""Parity of the four task bodies (C ABI) with the CPU oracle.

Each case runs the same seeded inputs through the GPU entry point and through
the oracle's restatement of the reference body; FP64 results must agree to
1e-12 relative (Frobenius), pivots exactly.
"""
import numpy as np
import pytest

from gpu_util import dev, host, ivec, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("n,c,ld", [(1, 1, 1), (7, 3, 9), (32, 16, 32), (33, 17, 40),
                                    (100, 1, 100), (256, 64, 300), (512, 592, 512),
                                    (1000, 40, 1003), (1024, 5, 1024)])
def test_leaf_solve(fs, oracle, cuda, n, c, ld):
    rng = np.random.default_rng(n * 1000 + c)
    D = rng.standard_normal((n, n)) / np.sqrt(n) + 2 * np.eye(n)
    X = rng.standard_normal((n, c))
    Dg, Xg, piv = dev(D, ld), dev(X, ld), ivec(n)
    assert fs.leaf_solve(Dg, Xg, piv) == 0
    Dr, Xr = np.asfortranarray(D.copy()), np.asfortranarray(X.copy())
    pr = np.zeros(n, dtype=np.int32)
    assert oracle.lib().ref_leaf_solve(n, c, oracle._p(Dr), n, oracle._p(Xr), n,
                                       pr.ctypes.data_as(oracle._ip)) == 0
    assert relerr(host(Xg), Xr) < TOL
    assert relerr(host(Dg), Dr) < TOL
    np.testing.assert_array_equal(piv.cpu().numpy()[:n], pr)


@pytest.mark.parametrize("n", [16, 100, 512])
def test_leaf_solve_needs_pivoting(fs, oracle, cuda, n):
    rng = np.random.default_rng(n)
    D = rng.standard_normal((n, n))  # no diagonal dominance: real interchanges
    X = rng.standard_normal((n, 9))
    Dg, Xg, piv = dev(D), dev(X), ivec(n)
    assert fs.leaf_solve(Dg, Xg, piv) == 0
    Dr, Xr = np.asfortranarray(D.copy()), np.asfortranarray(X.copy())
    pr = np.zeros(n, dtype=np.int32)
    oracle.lib().ref_leaf_solve(n, 9, oracle._p(Dr), n, oracle._p(Xr), n,
                                pr.ctypes.data_as(oracle._ip))
    np.testing.assert_array_equal(piv.cpu().numpy()[:n], pr)
    assert relerr(host(Dg), Dr) < 1e-11
    assert relerr(host(Xg), Xr) < 1e-10  # cond(D) ~ n for a Gaussian block


def test_leaf_solve_singular_reports_info(fs, oracle, cuda):
    n = 40
    D = np.eye(n)
    D[13, 13] = 0.0
    piv = ivec(n)
    info = fs.leaf_solve(dev(D), dev(np.ones((n, 2))), piv)
    Dr = np.asfortranarray(D.copy())
    Xr = np.asfortranarray(np.ones((n, 2)))
    assert info == oracle.lib().ref_leaf_solve(n, 2, oracle._p(Dr), n, oracle._p(Xr), n, None)
    assert info == 14


@pytest.mark.parametrize("k,r,ncol,col_beg", [(1, 1, 1, 0), (513, 30, 92, 2), (10000, 64, 80, 16),
                                               (131072, 64, 16, 0)])
def test_gemm_reduce(fs, oracle, cuda, k, r, ncol, col_beg):
    rng = np.random.default_rng(k + r)
    V = rng.standard_normal((k, r))
    U = rng.standard_normal((k, col_beg + ncol))
    W0 = rng.standard_normal((r, ncol))
    Vg, Ug, Wg = dev(V, k + 3), dev(U, k + 5), dev(W0, r + 1)
    fs.gemm_reduce(0.75, Vg, Ug, col_beg, ncol, Wg)
    Wr = np.asfortranarray(W0.copy())
    Vf, Uf = np.asfortranarray(V), np.asfortranarray(U)
    oracle.lib().ref_gemm_reduce(0.75, k, r, ncol, oracle._p(Vf), k, oracle._p(Uf), k, col_beg,
                                 oracle._p(Wr), r)
    assert relerr(host(Wg), Wr) < TOL


@pytest.mark.parametrize("k,r,c,u_col,d_col", [(1, 1, 1, 1, 0), (60, 30, 2, 62, 0),
                                                (512, 64, 528, 528, 0), (3000, 50, 358, 8, 58)])
def test_gemm_broadcast(fs, oracle, cuda, k, r, c, u_col, d_col):
    rng = np.random.default_rng(k * 7 + c)
    ncols = max(u_col + r, d_col + c)
    X = rng.standard_normal((k, ncols))
    eta = rng.standard_normal((r, c))
    Xg = dev(X, k + 2)
    fs.gemm_broadcast(-1.0, 1.0, Xg, u_col, r, dev(eta), d_col)
    Xr = np.asfortranarray(X.copy())
    etf = np.asfortranarray(eta)
    oracle.lib().ref_gemm_broadcast(-1.0, 1.0, k, r, c, oracle._p(Xr), k, u_col,
                                    oracle._p(etf), r, d_col)
    assert relerr(host(Xg), Xr) < TOL


@pytest.mark.parametrize("r,c", [(1, 1), (7, 3), (30, 92), (64, 592), (100, 40)])
@pytest.mark.parametrize("form", ["lu", "schur2"])
def test_node_solve(fs, oracle, cuda, r, c, form):
    if form == "schur2" and 2 * r > 144:
        pytest.skip("2r x 2r form is limited to 2r <= 144")
    rng = np.random.default_rng(r * 13 + c)
    V0Tu0 = 0.3 * rng.standard_normal((r, r)) / np.sqrt(r)
    V1Tu1 = 0.3 * rng.standard_normal((r, r)) / np.sqrt(r)
    V0Td0 = rng.standard_normal((r, c))
    V1Td1 = rng.standard_normal((r, c))
    g = [dev(V0Tu0, r + 1), dev(V1Tu1), dev(V0Td0, r + 2), dev(V1Td1)]
    fn = fs.node_lu_solve if form == "lu" else fs.node_schur2_solve
    assert fn(*g) == 0
    a = [np.asfortranarray(x.copy()) for x in (V0Tu0, V1Tu1, V0Td0, V1Td1)]
    ref = oracle.lib().ref_lu_node_solve if form == "lu" else oracle.lib().ref_schur2_solve
    assert ref(r, r, c, oracle._p(a[0]), r, oracle._p(a[1]), r, oracle._p(a[2]), r,
               oracle._p(a[3]), r) == 0
    assert relerr(host(g[2]), a[2]) < TOL
    assert relerr(host(g[3]), a[3]) < TOL


def test_node_solve_singular(fs, cuda):
    r = 5
    # S = I - V1Tu1 V0Tu0 = 0  when V1Tu1 = V0Tu0 = I
    g = [dev(np.eye(r)), dev(np.eye(r)), dev(np.ones((r, 2))), dev(np.ones((r, 2)))]
    assert fs.node_lu_solve(*g) > 0
