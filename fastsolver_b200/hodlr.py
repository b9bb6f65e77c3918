"""Python mirror of fastSolver's C++ interface over the native library.

Reference interface (paths relative to Charles-Chao-Chen/fastSolver):
  HodlrMatrix(col, row, gl, sl, r, t, leaf, name)   include/htree/hodlr_matrix.h:16-74
    .create_tree / .init_rhs / .init_circulant_matrix / .save_rhs /
    .save_solution / .get_num_leaf / .get_num_rhs / .launch_level
  FastSolver().bfs_solve(matrix, procs, ...)        include/solver/fast_solver.h:9-40
  gemm_reduce / gemm_broadcast / solve_node_matrix / leaf solve task bodies
                                                    include/solver/gemm.h:21-34,
                                                    include/solver/solver_tasks.h:13-23
The Legion context/runtime/Range arguments have no counterpart here: a system
lives on the current CUDA device and every call runs on one stream.  The
solver's additions (factor/solve split, mixed precision with FP64 refinement,
the HODLR matvec) are methods of the same classes.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import PREC_FP64, PREC_MIXED, NODE_FIELDS, call, check, lib

__all__ = ["HodlrMatrix", "FastSolver", "SystemBatch", "build_tree", "leaf_solve", "gemm_reduce",
           "gemm_broadcast", "node_lu_solve", "node_schur2_solve", "PREC_FP64", "PREC_MIXED"]


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(getattr(stream, "cuda_stream", 0)) or None


def build_tree(N: int, nrhs: int, rank: int, threshold: int) -> np.ndarray:
    """Node records (BFS order, NODE_FIELDS columns) of the tree HodlrMatrix
    builds; host only."""
    cap = 4 * (N // max(1, threshold // 2) + 2) + 8
    buf = (ctypes.c_int * (cap * len(NODE_FIELDS)))()
    nn = lib.hodlr_build_tree(N, nrhs, rank, threshold, buf, cap)
    check("hodlr_build_tree", 0 if nn > 0 else nn)
    return np.frombuffer(buf, dtype=np.int32)[: nn * len(NODE_FIELDS)].reshape(nn, -1).copy()


def _fortran(a: np.ndarray) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _ptr(a) -> int:
    """Device or host address of a torch tensor / numpy array."""
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    return int(a.ctypes.data)


def _ld(a) -> int:
    """Leading dimension of a column-major 2-D tensor/array (stride of dim 1)."""
    if hasattr(a, "stride"):
        st = a.stride()
        if a.dim() == 1:
            return max(1, a.shape[0])
        if st[0] != 1:
            raise ValueError("matrix must be column-major (stride(0) == 1)")
        return max(st[1], 1)
    if a.ndim == 1:
        return max(1, a.shape[0])
    if not a.flags.f_contiguous:
        raise ValueError("matrix must be Fortran-ordered")
    return max(a.shape[0], 1)


class HodlrMatrix:
    """A HODLR system on the current CUDA device.

    Mirrors HodlrMatrix(col, row, gl, sl, r, t, leaf, name): ``rhs_cols``
    right-hand sides, ``rhs_rows`` unknowns, ``rank`` at every level, dense
    leaves of at most ``threshold`` rows, ``leaf_size`` real leaves per
    Legion leaf (the reference's task granularity: it decides the drand48
    reseeding of init_rhs, the blocks of the text files and, for the FP64
    fused solve, which nodes use the 2r x 2r leaf-internal form).  The
    two-level launch (gl != sl) is the multi-GPU subtree split of
    fastsolver_b200.shard.
    """

    def __init__(self, rhs_cols: int, rhs_rows: int, rank: int, threshold: int,
                 leaf_size: int = 1, name: str = "global", glo_level: int | None = None,
                 sub_level: int | None = None):
        if int(leaf_size) < 1:
            raise ValueError("leaf_size must be >= 1")
        if glo_level is not None and sub_level is not None and glo_level != sub_level:
            raise NotImplementedError("two-level launch (gloLevel != subLevel): use "
                                      "fastsolver_b200.shard for the subtree split")
        self.rhs_cols, self.rhs_rows = int(rhs_cols), int(rhs_rows)
        self.rank, self.threshold = int(rank), int(threshold)
        self.leaf_size = int(leaf_size)
        self.file_rhs = name + "_rhs.txt"
        self.file_soln = name + "_soln.txt"
        self._h = None
        self._seed = 0

    # -- tree ---------------------------------------------------------------
    def create_tree(self) -> "HodlrMatrix":
        h = ctypes.c_void_p()
        call("hodlr_create", ctypes.byref(h), self.rhs_rows, self.rhs_cols, self.rank,
             self.threshold)
        self._h = h
        n, d, nl, nc, ml = (ctypes.c_int() for _ in range(5))
        call("hodlr_tree_info", self._h, ctypes.byref(n), ctypes.byref(d), ctypes.byref(nl),
             ctypes.byref(nc), ctypes.byref(ml))
        self.nnodes, self.max_depth, self.nleaves = n.value, d.value, nl.value
        self.ncols, self.max_leaf = nc.value, ml.value
        if self.leaf_size != 1:
            call("hodlr_set_leaf_size", self._h, self.leaf_size)
        return self

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("create_tree() first")
        return self._h

    def tree_nodes(self) -> np.ndarray:
        buf = (ctypes.c_int * (self.nnodes * len(NODE_FIELDS)))()
        call("hodlr_tree_nodes", self.handle, buf, self.nnodes)
        return np.frombuffer(buf, dtype=np.int32).reshape(self.nnodes, -1).copy()

    def get_num_leaf(self) -> int:
        """Legion leaves (tasks); equals the real leaves when leaf_size == 1."""
        n = lib.hodlr_get_num_leaf(self.handle)
        check("hodlr_get_num_leaf", min(n, 0))
        return n

    def legion_leaves(self) -> np.ndarray:
        """Node ids of the Legion leaves, left to right."""
        n = lib.hodlr_legion_leaves(self.handle, None, 0)
        buf = (ctypes.c_int * max(n, 1))()
        check("hodlr_legion_leaves", min(lib.hodlr_legion_leaves(self.handle, buf, n), 0))
        return np.array(buf[:n], dtype=np.int32)

    def get_num_rhs(self) -> int:
        return self.rhs_cols

    def launch_level(self) -> int:
        return 0

    # -- data -----------------------------------------------------------------
    def init_rhs(self, seed: int, stream=None):
        """drand48 right-hand side, reseeded per leaf (init_matrix_tasks.cc:43-77)."""
        self._seed = int(seed)
        call("hodlr_init_rhs_drand48", self.handle, int(seed), _stream_ptr(stream))

    def init_circulant_matrix(self, diag: float, stream=None):
        """diag*I + U U^T with U(i, j) = (i + j) mod r (the reference's test matrix)."""
        call("hodlr_init_circulant", self.handle, float(diag), _stream_ptr(stream))

    def init_gaussian(self, seed: int, offdiag_norm: float = 0.5, stream=None):
        call("hodlr_init_gaussian", self.handle, int(seed), float(offdiag_norm),
             _stream_ptr(stream))

    def set_matrix(self, D=None, U=None, V=None, stream=None):
        """Copy D (N x max_leaf), U, V (N x (C - m)) in; numpy (host) or torch CUDA."""
        host = int(any(x is not None and not hasattr(x, "data_ptr") for x in (D, U, V)))
        args = []
        keep = []
        for x in (D, U, V):
            if x is None:
                args += [None, 0]
            else:
                if not hasattr(x, "data_ptr"):
                    x = _fortran(x)
                keep.append(x)
                args += [_ptr(x), _ld(x)]
        call("hodlr_set_matrix", self.handle, *args, host, _stream_ptr(stream))

    def set_rhs(self, B, stream=None):
        host = int(not hasattr(B, "data_ptr"))
        if host:
            B = _fortran(B)
        call("hodlr_set_rhs", self.handle, _ptr(B), _ld(B), host, _stream_ptr(stream))

    def get_matrix(self, stream=None):
        """Host copies (D, U, V, B) of the system's data in the global layout."""
        N, vc = self.rhs_rows, self.ncols - self.rhs_cols
        D = np.zeros((N, self.max_leaf), order="F")
        U = np.zeros((N, max(vc, 0)), order="F")
        V = np.zeros((N, max(vc, 0)), order="F")
        B = np.zeros((N, self.rhs_cols), order="F")
        call("hodlr_get_matrix", self.handle, _ptr(D), N, _ptr(U) if vc else None, N,
             _ptr(V) if vc else None, N, _ptr(B), N, 1, _stream_ptr(stream))
        return D, U, V, B

    def solution(self, stream=None) -> np.ndarray:
        x = np.zeros((self.rhs_rows, self.rhs_cols), dtype=np.float64, order="F")
        call("hodlr_get_solution", self.handle, _ptr(x), self.rhs_rows, 1, _stream_ptr(stream))
        return x

    def solution_to(self, out, stream=None):
        """Device-to-device copy of the solution into a column-major torch tensor."""
        call("hodlr_get_solution", self.handle, _ptr(out), _ld(out), 0, _stream_ptr(stream))

    def matvec(self, x, y, stream=None):
        call("hodlr_matvec", self.handle, _ptr(x), _ld(x), _ptr(y), _ld(y), x.shape[1],
             _stream_ptr(stream))

    def relres(self, stream=None) -> float:
        out = ctypes.c_double()
        call("hodlr_relres", self.handle, ctypes.byref(out), _stream_ptr(stream))
        return out.value

    # -- launch schedule -------------------------------------------------------
    @property
    def schedule(self) -> dict:
        """The launch schedule (hodlr_schedule fields)."""
        c = _lib.Schedule()
        call("hodlr_get_schedule", self.handle, ctypes.byref(c))
        return c.as_dict()

    @schedule.setter
    def schedule(self, d: dict):
        cur = self.schedule
        cur.update(d)
        c = _lib.Schedule.from_dict(cur)
        call("hodlr_set_schedule", self.handle, ctypes.byref(c))

    def autotune(self, precision: int = PREC_MIXED, tol: float = 1e-12, reps: int = 2):
        """Time candidate schedules on the current matrix and RHS and keep the
        fastest; returns (schedule, ms per solve, [(schedule, ms), ...])."""
        return _tune(lambda *a: lib.hodlr_autotune(self.handle, int(precision), *a),
                     "hodlr_autotune", tol, reps)

    # -- per-phase device time ------------------------------------------------
    def set_profiling(self, on: bool):
        call("hodlr_set_profiling", self.handle, int(bool(on)))

    def phase_times(self, reset: bool = True) -> dict:
        """{phase: (ms, launches)} accumulated while profiling was on."""
        ms = (ctypes.c_double * len(_lib.PHASES))()
        ln = (ctypes.c_longlong * len(_lib.PHASES))()
        call("hodlr_phase_times", self.handle, ms, ln, int(reset))
        return {k: (ms[i], int(ln[i])) for i, k in enumerate(_lib.PHASES)}

    # -- reference text format (save_region_task.cc:37-67) -------------------
    def save_solution(self, filename: str | None = None):
        """HodlrMatrix::save_solution (hodlr_matrix.cc:581-590)."""
        call("hodlr_save_solution", self.handle, (filename or self.file_soln).encode())

    def save_rhs(self, filename: str | None = None, seed: int | None = None):
        """HodlrMatrix::save_rhs (hodlr_matrix.cc:569-579): one seed line per Legion leaf."""
        sd = self._seed if seed is None else int(seed)
        call("hodlr_save_rhs", self.handle, (filename or self.file_rhs).encode(), sd)

    def load_rhs(self, filename: str | None = None) -> int:
        """Read a right-hand-side file in save_rhs's format into b; returns its seed."""
        sd = ctypes.c_long()
        call("hodlr_load_rhs", self.handle, (filename or self.file_rhs).encode(),
             ctypes.byref(sd))
        self._seed = int(sd.value)
        return self._seed

    def close(self):
        if self._h is not None:
            lib.hodlr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FastSolver:
    """Mirrors FastSolver (include/solver/fast_solver.h:9-40)."""

    def bfs_solve(self, matrix: HodlrMatrix, schur2: bool = False, sync: bool = True,
                  stream=None) -> int:
        """Fused FP64 factor+solve of the current RHS, as the reference's bfs_solve."""
        return call("hodlr_solve_fused", matrix.handle, int(schur2), int(sync),
                    _stream_ptr(stream))

    def factor(self, matrix: HodlrMatrix, precision: int = PREC_FP64, stream=None):
        call("hodlr_factor", matrix.handle, int(precision), _stream_ptr(stream))

    def solve(self, matrix: HodlrMatrix, stream=None):
        call("hodlr_solve", matrix.handle, _stream_ptr(stream))

    def solve_refined(self, matrix: HodlrMatrix, precision: int = PREC_MIXED,
                      tol: float = 1e-12, maxiter: int = 10, stream=None, check_conv=True):
        it = ctypes.c_int()
        rr = ctypes.c_double()
        st = lib.hodlr_solve_refined(matrix.handle, int(precision), float(tol), int(maxiter),
                                     ctypes.byref(it), ctypes.byref(rr), _stream_ptr(stream))
        if check_conv or st != _lib.ERR_NOCONV:
            check("hodlr_solve_refined", st)
        return it.value, rr.value

    def solve_refined_host(self, matrix: HodlrMatrix, D, U, V, B, out=None,
                           precision: int = PREC_MIXED, tol: float = 1e-12, maxiter: int = 10,
                           stream=None, check_conv=True):
        """Host-to-host refined solve: D, U, V, B are column-major host arrays
        (numpy, or pinned CPU torch tensors for overlapped copies), `out` an
        optional column-major host array (N x nrhs) for the solution.  Returns
        (x, sweeps, relres)."""
        ins = [x if hasattr(x, "data_ptr") else _fortran(x) for x in (D, U, V, B)]
        if out is None:
            out = np.zeros((matrix.rhs_rows, matrix.rhs_cols), dtype=np.float64, order="F")
        it = ctypes.c_int()
        rr = ctypes.c_double()
        args = []
        for x in ins:
            args += [_ptr(x), _ld(x)]
        st = lib.hodlr_solve_refined_host(matrix.handle, *args, _ptr(out), _ld(out),
                                          int(precision), float(tol), int(maxiter),
                                          ctypes.byref(it), ctypes.byref(rr), _stream_ptr(stream))
        if check_conv or st != _lib.ERR_NOCONV:
            check("hodlr_solve_refined_host", st)
        return out, it.value, rr.value


def _tune(fn, name, tol, reps, cap=64):
    best = _lib.Schedule()
    ms = ctypes.c_double()
    log = (_lib.TuneTrial * cap)()
    n = ctypes.c_int()
    check(name, fn(float(tol), int(reps), ctypes.byref(best), ctypes.byref(ms), log, cap,
                   ctypes.byref(n)))
    trials = [(log[i].schedule.as_dict(), log[i].ms) for i in range(min(n.value, cap))]
    return best.as_dict(), ms.value, trials


class SystemBatch:
    """Independent HODLR systems of uneven size, rank, leaf size and RHS count
    solved together (one merged launch per tree level and phase).  The
    matrices keep their own data: load matrices and RHS into them as usual,
    call solve_refined, then read each matrix's solution().  The matrices must
    stay open while the batch exists."""

    def __init__(self, matrices):
        self.matrices = list(matrices)
        arr = (ctypes.c_void_p * len(self.matrices))(*[m.handle.value for m in self.matrices])
        h = ctypes.c_void_p()
        call("hodlr_batch_create", ctypes.byref(h), arr, len(self.matrices))
        self._h = h

    def solve_refined(self, tol: float = 1e-12, maxiter: int = 10, stream=None,
                      check_conv=True):
        """Returns (sweeps, per-system relative residuals)."""
        it, mx, failed = ctypes.c_int(), ctypes.c_double(), ctypes.c_int(-1)
        rr = (ctypes.c_double * len(self.matrices))()
        st = lib.hodlr_batch_solve_refined(self._h, float(tol), int(maxiter), ctypes.byref(it),
                                           ctypes.byref(mx), rr, ctypes.byref(failed),
                                           _stream_ptr(stream))
        self.failed = failed.value
        if check_conv or st != _lib.ERR_NOCONV:
            check("hodlr_batch_solve_refined", st)
        return it.value, list(rr)

    def autotune(self, tol: float = 1e-12, reps: int = 2):
        """One schedule for all systems, timed as the batched solve; returns
        (schedule, ms per batched solve, [(schedule, ms), ...])."""
        return _tune(lambda *a: lib.hodlr_batch_autotune(self._h, *a), "hodlr_batch_autotune",
                     tol, reps)

    def set_profiling(self, on: bool):
        call("hodlr_batch_set_profiling", self._h, int(bool(on)))

    def phase_times(self, reset: bool = True) -> dict:
        ms = (ctypes.c_double * len(_lib.PHASES))()
        ln = (ctypes.c_longlong * len(_lib.PHASES))()
        call("hodlr_batch_phase_times", self._h, ms, ln, int(reset))
        return {k: (ms[i], int(ln[i])) for i, k in enumerate(_lib.PHASES)}

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib.hodlr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# task bodies on column-major torch CUDA tensors
# ---------------------------------------------------------------------------

def leaf_solve(D, X, ipiv, info=None, stream=None) -> int:
    n = D.shape[0]
    return call("hodlr_leaf_solve", n, X.shape[1], _ptr(D), _ld(D), _ptr(X), _ld(X), _ptr(ipiv),
                _ptr(info) if info is not None else None, _stream_ptr(stream),
                ok=tuple([0] + list(range(1, n + 1))))


def gemm_reduce(alpha, V, U, col_beg, ncol, W, stream=None):
    k, r = V.shape
    call("hodlr_gemm_reduce", float(alpha), k, r, ncol, _ptr(V), _ld(V), _ptr(U), _ld(U),
         col_beg, _ptr(W), _ld(W), _stream_ptr(stream))


def gemm_broadcast(alpha, beta, X, u_col_beg, r, eta, d_col_beg, stream=None):
    k = X.shape[0]
    c = eta.shape[1]
    call("hodlr_gemm_broadcast", float(alpha), float(beta), k, r, c, _ptr(X), _ld(X), u_col_beg,
         _ptr(eta), _ld(eta), d_col_beg, _stream_ptr(stream))


def _node(fn, V0Tu0, V1Tu1, V0Td0, V1Td1, info, stream):
    r1, r0 = V0Tu0.shape
    c = V0Td0.shape[1]
    return call(fn, r0, r1, c, _ptr(V0Tu0), _ld(V0Tu0), _ptr(V1Tu1), _ld(V1Tu1), _ptr(V0Td0),
                _ld(V0Td0), _ptr(V1Td1), _ld(V1Td1),
                _ptr(info) if info is not None else None, _stream_ptr(stream),
                ok=tuple(range(0, r0 + r1 + 1)))


def node_lu_solve(V0Tu0, V1Tu1, V0Td0, V1Td1, info=None, stream=None) -> int:
    return _node("hodlr_node_lu_solve", V0Tu0, V1Tu1, V0Td0, V1Td1, info, stream)


def node_schur2_solve(V0Tu0, V1Tu1, V0Td0, V1Td1, info=None, stream=None) -> int:
    return _node("hodlr_node_schur2_solve", V0Tu0, V1Tu1, V0Td0, V1Td1, info, stream)


def write_text(filename: str, X, col_beg: int = 0, ncol: int | None = None, seed: int = 0,
               print_seed: bool = False):
    """Append X's rows (columns col_beg.. of a 2-D array) in the reference's
    text format (save_data, save_region_task.cc:37-67)."""
    A = np.asfortranarray(np.asarray(X, dtype=np.float64))
    nrow, cols = A.shape
    ncol = cols - col_beg if ncol is None else int(ncol)
    call("hodlr_text_write", filename.encode(), A.ctypes.data, max(nrow, 1), nrow,
         int(col_beg), ncol, int(seed), int(bool(print_seed)))


def read_text(filename: str, nrow: int, ncol: int, block_rows=None):
    """Read an nrow x ncol block written in the reference's text format.

    Without ``block_rows`` the file holds the values only (a solution file,
    read as direct_solve.cc:201-213 does); with it, one seed line precedes
    each block of block_rows[b] rows (a right-hand-side file).  Returns
    (X, seeds)."""
    X = np.zeros((nrow, ncol), dtype=np.float64, order="F")
    if block_rows is None:
        call("hodlr_text_read", filename.encode(), X.ctypes.data, max(nrow, 1), nrow, ncol, 0,
             None, None)
        return X, []
    br = (ctypes.c_int * len(block_rows))(*[int(b) for b in block_rows])
    sd = (ctypes.c_long * max(len(block_rows), 1))()
    call("hodlr_text_read", filename.encode(), X.ctypes.data, max(nrow, 1), nrow, ncol,
         len(block_rows), br, sd)
    return X, [int(v) for v in sd[:len(block_rows)]]
