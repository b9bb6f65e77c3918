"""ctypes front end of the CPU oracle (oracle/refcpu.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product path
(fastsolver_b200) never imports this module.

The C library restates fastSolver's FP64 CPU path (src/solver/solver_tasks.cc,
src/solver/gemm.cc, src/solver/fast_solver.cc, src/htree/hodlr_matrix.cc);
each C function names the reference lines it follows.  This module adds the
system builders the tests feed to both the oracle and the GPU:

* ``kat_system``: the reference's only test matrix, A = diag*I + U U^T with
  circulant U(i, j) = (i + j) mod r and a drand48 RHS reseeded per leaf
  (test/single_launch.cc:20-75, init_matrix_tasks.cc:43-77/176-219,
  hodlr_matrix.cc:528-567).
* ``gaussian_system``: the synthetic distribution of the benchmark configs
  (leaf blocks G/sqrt(n) + 2I, U/V iid N(0,1)/sqrt(r*n_child) rescaled so each
  off-diagonal block U_c V_s^T has spectral norm 0.5, b iid N(0,1)), drawn with
  numpy's PCG64 from a seed.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

FIELDS = ["nrow", "ncol", "row_beg", "col_beg", "lchild", "rchild", "parent",
          "depth", "vncol", "is_leaf"]
F = {k: i for i, k in enumerate(FIELDS)}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def blas_path() -> str:
    """Path of the OpenBLAS that scipy bundles (exports scipy_dgemm_/dgesv_)."""
    import scipy  # noqa: F401  (locates site-packages)
    base = os.path.dirname(os.path.dirname(scipy.__file__))
    hits = sorted(glob.glob(os.path.join(base, "scipy.libs", "libscipy_openblas*.so")))
    if not hits:
        raise RuntimeError("scipy's bundled OpenBLAS was not found")
    return hits[0]


def build(force: bool = False) -> str:
    so = os.path.join(_HERE, "librefcpu.so")
    src = os.path.join(_HERE, "refcpu.c")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-o", so, src,
                               "-ldl", "-lm"])
    return so


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    so = os.path.join(_HERE, "librefcpu.so")
    if not os.path.exists(so):
        build()
    L = ctypes.CDLL(so)
    L.ref_load_blas.argtypes = [ctypes.c_char_p]
    rc = L.ref_load_blas(blas_path().encode())
    if rc != 0:
        raise RuntimeError(f"ref_load_blas failed ({rc})")
    L.ref_build_tree.argtypes = [ctypes.c_int] * 4 + [_ip, ctypes.c_int]
    L.ref_leaf_solve.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                 ctypes.c_int, _ip]
    L.ref_gemm_reduce.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _dp,
                                  ctypes.c_int]
    L.ref_gemm_broadcast.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                     ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int]
    for fn in (L.ref_lu_node_solve, L.ref_schur2_solve):
        fn.argtypes = [ctypes.c_int] * 3 + [_dp, ctypes.c_int] * 4
    L.ref_bfs_solve.argtypes = [_ip, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int,
                                _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.ref_bfs_solve_ls.argtypes = [_ip, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int,
                                   _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.ref_hodlr_matvec.argtypes = [_ip, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int,
                                   _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int,
                                   ctypes.c_int]
    L.ref_hodlr_dense.argtypes = [_ip, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int,
                                  _dp, ctypes.c_int, _dp, ctypes.c_int]
    L.ref_drand48_fill.argtypes = [ctypes.c_long, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
    L.ref_fill_circulant_u.argtypes = [ctypes.c_int] * 5 + [_dp, ctypes.c_int]
    L.ref_fill_circulant_k.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, _dp, ctypes.c_int]
    L.ref_dense_solve.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                  ctypes.c_int]
    L.ref_rel_error.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                ctypes.c_int]
    L.ref_rel_error.restype = ctypes.c_double
    L.ref_set_blas_threads.argtypes = [ctypes.c_int]
    _LIB = L
    return L


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(_dp)


def _ld(a: np.ndarray) -> int:
    return a.shape[0] if a.ndim == 2 else a.shape[0]


def fmat(rows: int, cols: int) -> np.ndarray:
    return np.zeros((rows, max(cols, 0)), dtype=np.float64, order="F")


# --------------------------------------------------------------------------
# tree
# --------------------------------------------------------------------------

def build_tree(N: int, nrhs: int, rank: int, threshold: int) -> np.ndarray:
    cap = 4 * (N // max(1, threshold // 2) + 2) + 8
    buf = np.zeros(cap * len(FIELDS), dtype=np.int32)
    nn = lib().ref_build_tree(N, nrhs, rank, threshold, buf.ctypes.data_as(_ip), cap)
    if nn < 0:
        raise ValueError(f"ref_build_tree failed ({nn})")
    return buf[: nn * len(FIELDS)].reshape(nn, len(FIELDS)).copy()


def leaves(tree: np.ndarray):
    return [i for i in range(tree.shape[0]) if tree[i, F["is_leaf"]]]


def total_cols(tree: np.ndarray) -> int:
    """Columns of X: max over leaves of col_beg + ncol (root: nrhs)."""
    return int(max(tree[i, F["col_beg"]] + tree[i, F["ncol"]] for i in leaves(tree)))


def max_leaf(tree: np.ndarray) -> int:
    return int(max(tree[i, F["nrow"]] for i in leaves(tree)))


# --------------------------------------------------------------------------
# systems
# --------------------------------------------------------------------------

class System:
    """A HODLR system in the global layout the oracle and the GPU share.

    D (N x nmax): leaf blocks stacked; U, V (N x C-m): factors by column block;
    B (N x m): right-hand sides.  ``X0()`` returns the solver's working array
    [b | U] (U restricted, per leaf, to its ancestors' column blocks).
    """

    def __init__(self, tree, D, U, V, B):
        self.tree, self.D, self.U, self.V, self.B = tree, D, U, V, B
        self.N = int(tree[0, F["nrow"]])
        self.m = int(tree[0, F["ncol"]])
        self.C = total_cols(tree)

    def X0(self) -> np.ndarray:
        X = fmat(self.N, self.C)
        X[:, : self.m] = self.B
        t = self.tree
        for i in leaves(t):
            rb, n = t[i, F["row_beg"]], t[i, F["nrow"]]
            cend = t[i, F["col_beg"]] + t[i, F["ncol"]]
            X[rb:rb + n, self.m:cend] = self.U[rb:rb + n, : cend - self.m]
        return X

    def dense(self) -> np.ndarray:
        A = fmat(self.N, self.N)
        t = np.ascontiguousarray(self.tree, dtype=np.int32)
        lib().ref_hodlr_dense(t.ctypes.data_as(_ip), t.shape[0], _p(self.D), self.D.shape[0],
                              _p(self.U), self.U.shape[0], _p(self.V), self.V.shape[0],
                              _p(A), A.shape[0])
        return A


def legion_leaves(tree: np.ndarray, leaf_size: int = 1):
    """Topmost nodes with at most leaf_size real leaves below, left to right
    (mark_legion_leaf, hodlr_matrix.cc:317-337)."""
    def nreal(i):
        if tree[i, F["is_leaf"]]:
            return 1
        return nreal(int(tree[i, F["lchild"]])) + nreal(int(tree[i, F["rchild"]]))

    out = []

    def walk(i):
        if nreal(i) <= leaf_size:
            out.append(i)
            return
        walk(int(tree[i, F["lchild"]]))
        walk(int(tree[i, F["rchild"]]))

    walk(0)
    return out


def kat_system(N=480, nrhs=2, rank=30, threshold=60, diag=1.0e4, seed=1245667,
               leaf_size=1) -> System:
    """The reference's accuracy run (test/single_launch.cc:20-75); the drand48
    right-hand side is reseeded per Legion leaf (init_rhs_recursive,
    hodlr_matrix.cc:191-209)."""
    L = lib()
    tree = build_tree(N, nrhs, rank, threshold)
    C = total_cols(tree)
    nmax = max_leaf(tree)
    D = fmat(N, nmax)
    U = fmat(N, C - nrhs)
    V = fmat(N, C - nrhs)
    B = fmat(N, nrhs)
    for i in leaves(tree):
        rb, n = int(tree[i, F["row_beg"]]), int(tree[i, F["nrow"]])
        blk = fmat(n, nmax)
        L.ref_fill_circulant_k(n, rb, rank, diag, _p(blk), n)
        D[rb:rb + n, :] = blk
    for i in legion_leaves(tree, leaf_size):
        rb, n = int(tree[i, F["row_beg"]]), int(tree[i, F["nrow"]])
        bb = fmat(n, nrhs)
        L.ref_drand48_fill(seed, n, nrhs, _p(bb), n)
        B[rb:rb + n, :] = bb
    # U and V: circulant (i + j) % r in global rows, every level the same
    Ublk = fmat(N, rank)
    L.ref_fill_circulant_u(N, rank, 0, 0, rank, _p(Ublk), N)
    for lvl in range((C - nrhs) // rank):
        U[:, lvl * rank:(lvl + 1) * rank] = Ublk
        V[:, lvl * rank:(lvl + 1) * rank] = Ublk
    return System(tree, D, U, V, B)


def _spectral_norm_uv(Uc: np.ndarray, Vs: np.ndarray) -> float:
    gu = Uc.T @ Uc
    gv = Vs.T @ Vs
    w = np.linalg.eigvals(gu @ gv)
    return float(np.sqrt(np.max(np.abs(w.real))))


def gaussian_system(N, nrhs, rank, threshold, seed=1245667, offdiag_norm=0.5) -> System:
    """Synthetic system with the benchmark configs' value distributions."""
    rng = np.random.default_rng(seed)
    tree = build_tree(N, nrhs, rank, threshold)
    C = total_cols(tree)
    nmax = max_leaf(tree)
    D = fmat(N, nmax)
    U = fmat(N, C - nrhs)
    V = fmat(N, C - nrhs)
    for i in leaves(tree):
        rb, n = int(tree[i, F["row_beg"]]), int(tree[i, F["nrow"]])
        G = rng.standard_normal((n, n))
        D[rb:rb + n, :n] = G / np.sqrt(n) + 2.0 * np.eye(n)
    m = nrhs
    for p in range(tree.shape[0]):
        if tree[p, F["is_leaf"]]:
            continue
        kids = [int(tree[p, F["lchild"]]), int(tree[p, F["rchild"]])]
        for c in kids:
            rb, n = int(tree[c, F["row_beg"]]), int(tree[c, F["nrow"]])
            off = int(tree[c, F["col_beg"]]) - m
            r = int(tree[c, F["ncol"]])
            U[rb:rb + n, off:off + r] = rng.standard_normal((n, r)) / np.sqrt(r * n)
            V[rb:rb + n, off:off + r] = rng.standard_normal((n, r)) / np.sqrt(r * n)
        for c, s in ((kids[0], kids[1]), (kids[1], kids[0])):
            rbc, nc = int(tree[c, F["row_beg"]]), int(tree[c, F["nrow"]])
            rbs, ns = int(tree[s, F["row_beg"]]), int(tree[s, F["nrow"]])
            oc = int(tree[c, F["col_beg"]]) - m
            os_ = int(tree[s, F["col_beg"]]) - m
            r = int(tree[c, F["ncol"]])
            Uc = U[rbc:rbc + nc, oc:oc + r]
            Vs = V[rbs:rbs + ns, os_:os_ + r]
            nrm = _spectral_norm_uv(Uc, Vs)
            s_ = np.sqrt(offdiag_norm / nrm)
            U[rbc:rbc + nc, oc:oc + r] *= s_
            V[rbs:rbs + ns, os_:os_ + r] *= s_
    B = np.asfortranarray(rng.standard_normal((N, nrhs)))
    return System(tree, D, U, V, B)


# --------------------------------------------------------------------------
# solves
# --------------------------------------------------------------------------

def bfs_solve(sysm: System, nthreads: int = 1, schur2: bool = False, leaf_size: int = 1):
    """Fused FP64 solve (fast_solver.cc:136-255); leaf_size > 1 solves the
    nodes inside a Legion leaf with the 2r x 2r form. Returns (X, D_lu)."""
    L = lib()
    X = sysm.X0()
    D = np.asfortranarray(sysm.D.copy())
    t = np.ascontiguousarray(sysm.tree, dtype=np.int32)
    L.ref_set_blas_threads(1)
    rc = L.ref_bfs_solve_ls(t.ctypes.data_as(_ip), t.shape[0], _p(X), X.shape[0],
                            _p(sysm.V), sysm.V.shape[0], _p(D), D.shape[0], nthreads,
                            1 if schur2 else 0, int(leaf_size))
    if rc != 0:
        raise RuntimeError(f"ref_bfs_solve INFO={rc}")
    return X, D


def matvec(sysm: System, x: np.ndarray) -> np.ndarray:
    x = np.asfortranarray(x, dtype=np.float64)
    m = x.shape[1]
    y = fmat(sysm.N, m)
    t = np.ascontiguousarray(sysm.tree, dtype=np.int32)
    lib().ref_hodlr_matvec(t.ctypes.data_as(_ip), t.shape[0], _p(sysm.D), sysm.D.shape[0],
                           _p(sysm.U), sysm.U.shape[0], _p(sysm.V), sysm.V.shape[0],
                           _p(x), x.shape[0], _p(y), y.shape[0], m)
    return y


def dense_solve(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    A = np.asfortranarray(A.copy())
    X = np.asfortranarray(B.copy())
    rc = lib().ref_dense_solve(A.shape[0], X.shape[1], _p(A), A.shape[0], _p(X), X.shape[0])
    if rc != 0:
        raise RuntimeError(f"dense dgesv INFO={rc}")
    return X


def rel_error(x: np.ndarray, xref: np.ndarray) -> float:
    x = np.asfortranarray(x, dtype=np.float64)
    xref = np.asfortranarray(xref, dtype=np.float64)
    return float(lib().ref_rel_error(x.shape[0], x.shape[1], _p(x), x.shape[0], _p(xref),
                                     xref.shape[0]))


def relres(sysm: System, x: np.ndarray) -> float:
    """max_j ||b_j - A x_j||_2 / ||b_j||_2 through the HODLR matvec."""
    r = sysm.B - matvec(sysm, x)
    return float(np.max(np.linalg.norm(r, axis=0) / np.linalg.norm(sysm.B, axis=0)))
