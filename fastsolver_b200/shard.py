"""Subtree sharding of one HODLR system over several GPUs (one process each).

The reference splits a solve the same way (test/parallel_launch.cc:20-110,
test/sub_solve_task.cc:59-112, FastSolver::solve_top / solve_top_bfs /
visit_const in src/solver/fast_solver.cc:74-134, 257-322): the nodes at depth
k = log2(P) of the global tree root P independent subtrees; each part solves
its subtree as a HODLR system of its own whose right-hand side carries, next
to b, the U blocks of its k ancestors (the sub-problem's root has
nrhs + rank * k columns, sub_solve_task.cc:87); then the top k levels are
walked bottom-up over the parts' results.

Here every part is one process with its own GPU.  Below depth k a part's
sub-solve is the ordinary fused FP64 solve of its rows (no communication).
For a top-level node P with children c0, c1 the reduce V_c^T [d_c | u_c] runs
on every part's own rows of c and the partial sums are added by one
all-reduce per level (NCCL on GPUs; the REDOP_ADD reduction of gemm.cc:74-133
across parts); every part then solves P's capacitance system itself (a few
r x r blocks) and applies the broadcast d_c -= u_c eta to its own rows.  The
exchange per level is 2^d * 2 * r * (m + r (d + 1)) doubles (about 80 KB at
the root for r = 64, m = 16): no bulk data crosses the GPUs.

The task bodies are pluggable (``bodies``); the default runs the library's
C ABI on the current CUDA device (the sub-solve through hodlr_solve_fused,
the top levels through hodlr_gemm_reduce, hodlr_node_lu_solve and
hodlr_gemm_broadcast).
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import NODE_FIELDS

F = {k: i for i, k in enumerate(NODE_FIELDS)}


class SubtreeSplit:
    """Partition of the global tree into ``nparts`` subtrees (a power of two):
    the nodes at depth k = log2(nparts), left to right; part g owns the rows
    of its subtree and walks the top path of its k ancestors."""

    def __init__(self, N: int, nrhs: int, rank: int, threshold: int, nparts: int,
                 tree: np.ndarray | None = None):
        if nparts < 1 or nparts & (nparts - 1):
            raise ValueError("the number of parts must be a power of two")
        if tree is None:
            from .hodlr import build_tree
            tree = build_tree(N, nrhs, rank, threshold)
        self.tree = np.asarray(tree)
        self.N, self.m, self.r, self.threshold = int(N), int(nrhs), int(rank), int(threshold)
        self.nparts = int(nparts)
        self.k = int(round(math.log2(nparts)))   # launch level
        t = self.tree
        frontier = [0]
        for _ in range(self.k):
            nxt = []
            for i in frontier:
                if t[i, F["is_leaf"]]:
                    raise ValueError(f"the tree is too shallow for {nparts} parts")
                nxt += [int(t[i, F["lchild"]]), int(t[i, F["rchild"]])]
            frontier = nxt
        self.roots = frontier                     # sub-root node ids, left to right
        self.C = int(max(t[i, F["col_beg"]] + t[i, F["ncol"]]
                         for i in range(t.shape[0]) if t[i, F["is_leaf"]]))

    # -- per part ---------------------------------------------------------------
    def rows(self, g: int) -> tuple[int, int]:
        i = self.roots[g]
        return int(self.tree[i, F["row_beg"]]), int(self.tree[i, F["nrow"]])

    def sub_shape(self, g: int) -> tuple[int, int, int, int]:
        """(N_g, nrhs_g, rank, threshold) of part g's HODLR sub-system."""
        return self.rows(g)[1], self.m + self.r * self.k, self.r, self.threshold

    def ancestors(self, g: int):
        """[(P, c, side)] from depth k - 1 up to the root: the top-level node P
        at each depth, its child c on part g's side and which child it is."""
        t = self.tree
        out = []
        c = self.roots[g]
        while c != 0:
            P = int(t[c, F["parent"]])
            out.append((P, c, 0 if int(t[P, F["lchild"]]) == c else 1))
            c = P
        return out

    def local_arrays(self, g: int, D, U, V, B):
        """Part g's slices of the global layout: D rows; U, V columns of the
        subtree's own levels (depth > k); b next to the U blocks of the k top
        levels (the sub-problem's right-hand side).  Also returns the V blocks
        of the top levels (rows of part g), one r-column block per depth."""
        rb, n = self.rows(g)
        rk = self.r * self.k
        rs = slice(rb, rb + n)
        Dg = np.asfortranarray(D[rs, :])
        Ug = np.asfortranarray(U[rs, rk:])
        Vg = np.asfortranarray(V[rs, rk:])
        Bg = np.asfortranarray(np.concatenate([B[rs, :], U[rs, :rk]], axis=1))
        Vtop = np.asfortranarray(V[rs, :rk])
        return Dg, Ug, Vg, Bg, Vtop

    def level_slot(self, d: int, P: int, side: int) -> int:
        """Index of (node P at depth d, child side) in the level's exchange buffer."""
        at_d = [i for i in range(self.tree.shape[0]) if int(self.tree[i, F["depth"]]) == d]
        return 2 * at_d.index(P) + side


class GpuBodies:
    """The task bodies on the current CUDA device, through the C ABI."""

    def __init__(self, stream=None):
        import torch
        self.torch = torch
        self.stream = stream
        self.dev = torch.device("cuda", torch.cuda.current_device())

    def _colmajor(self, a):
        t = self.torch
        a = np.asarray(a, dtype=np.float64)
        x = t.empty((a.shape[1], a.shape[0]), dtype=t.float64, device=self.dev).T
        x.copy_(t.from_numpy(np.ascontiguousarray(a)))
        return x

    def zeros(self, rows, cols):
        t = self.torch
        return t.zeros((cols, rows), dtype=t.float64, device=self.dev).T

    def sub_solve(self, shape, Dg, Ug, Vg, Bg):
        """Fused FP64 solve of the part's sub-system; X (N_g x nrhs_g) on the device."""
        from .hodlr import FastSolver, HodlrMatrix
        n, nrhs, r, thr = shape
        h = HodlrMatrix(nrhs, n, r, thr).create_tree()
        h.set_matrix(Dg, Ug if Ug.shape[1] else None, Vg if Vg.shape[1] else None,
                     stream=self.stream)
        h.set_rhs(Bg, stream=self.stream)
        FastSolver().bfs_solve(h, stream=self.stream)
        X = self.zeros(n, nrhs)
        h.solution_to(X, stream=self.stream)
        self.torch.cuda.synchronize()
        h.close()
        return X

    def upload(self, a):
        return self._colmajor(a)

    def reduce(self, V, X, ncol):
        """W = V^T X[:, :ncol] (gemm.cc:315-384 into a zeroed region)."""
        from .hodlr import gemm_reduce
        W = self.zeros(V.shape[1], ncol)
        gemm_reduce(1.0, V, X, 0, ncol, W, stream=self.stream)
        return W

    def node_solve(self, W0, W1, cw):
        """LUSolveTask (solver_tasks.cc:139-305) on the summed reduce results;
        returns (eta0, eta1), the right-hand sides of children 0 and 1."""
        from .hodlr import node_lu_solve
        V0Td0, V0Tu0 = W0[:, :cw].clone(), W0[:, cw:].clone()
        V1Td1, V1Tu1 = W1[:, :cw].clone(), W1[:, cw:].clone()
        info = node_lu_solve(V0Tu0, V1Tu1, V0Td0, V1Td1, stream=self.stream)
        if info:
            raise RuntimeError(f"node solve INFO={info}")
        return V1Td1, V0Td0   # fast_solver.cc:238-240: eta0 = V1Td1, eta1 = V0Td0

    def broadcast(self, X, u_col_beg, r, eta, ncol):
        """X[:, :ncol] -= X[:, u_col_beg:u_col_beg + r] eta (gemm.cc:417-478)."""
        from .hodlr import gemm_broadcast
        gemm_broadcast(-1.0, 1.0, X, u_col_beg, r, eta, 0, stream=self.stream)

    def to_exchange(self, W):
        return W

    def from_exchange(self, buf):
        return buf

    def exchange_buffer(self, nslots, rows, cols):
        t = self.torch
        return t.zeros((nslots, cols, rows), dtype=t.float64, device=self.dev)

    def host(self, X):
        return X.detach().cpu().numpy()


class TorchComm:
    """All-reduce (sum) over a torch.distributed process group.  With the gloo
    backend the buffer goes through host memory; with NCCL it stays on the GPU."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.gloo = dist.get_backend(group) == "gloo"

    def allreduce_sum(self, buf):
        if self.gloo and getattr(buf, "is_cuda", False):
            h = buf.cpu()
            self.dist.all_reduce(h, group=self.group)
            buf.copy_(h)
        else:
            self.dist.all_reduce(buf, group=self.group)
        return buf


class ShardedSolver:
    """Part g's side of the sharded fused FP64 solve (the reference's
    SubSolveTask + FastSolver::solve_top)."""

    def __init__(self, split: SubtreeSplit, part: int, comm, bodies=None):
        self.split, self.g, self.comm = split, int(part), comm
        self.bodies = bodies if bodies is not None else GpuBodies()

    def solve(self, Dg, Ug, Vg, Bg, Vtop):
        """Returns part g's rows of the solution (N_g x m).  Every part must
        call this together: the top levels all-reduce once per level."""
        sp, b = self.split, self.bodies
        m, r = sp.m, sp.r
        X = b.sub_solve(sp.sub_shape(self.g), Dg, Ug, Vg, Bg)   # A_sub^{-1} [b | U_top]
        Vt = b.upload(Vtop) if Vtop.shape[1] else None
        for (P, c, side) in sp.ancestors(self.g):
            d = int(sp.tree[P, F["depth"]])
            cw = m + r * d                       # columns [0, c.col_beg) carried up
            ncol = cw + r                        # [d_c | u_c]
            V_c = Vt[:, r * d: r * (d + 1)]      # V block of child c, part g's rows
            W = b.reduce(V_c, X, ncol)           # partial V_c^T [d_c | u_c]
            nslots = 2 * (1 << d)
            buf = b.exchange_buffer(nslots, r, ncol)
            buf[sp.level_slot(d, P, side)] = b.to_exchange(W).T
            self.comm.allreduce_sum(buf)
            s0 = sp.level_slot(d, P, 0)
            W0, W1 = b.from_exchange(buf[s0].T), b.from_exchange(buf[s0 + 1].T)
            eta0, eta1 = b.node_solve(W0, W1, cw)
            b.broadcast(X, cw, r, eta0 if side == 0 else eta1, cw)
        return b.host(X[:, :m])
