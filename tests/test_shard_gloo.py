"""Subtree sharding of one system over 2 and 4 processes (gloo, CPU).

Each process is one part of fastsolver_b200.shard: it solves its subtree as a
HODLR sub-system whose right-hand side carries the U blocks of its top
ancestors, then walks the top levels, adding the parts' partial reduces with
one all-reduce per level.  Here the task bodies are the oracle's restated
reference bodies on the CPU (sub-solve = the oracle's fused FP64 walk of the
sub-system, reduce / LUSolve / broadcast = ref_gemm_reduce /
ref_lu_node_solve / ref_gemm_broadcast), so the test checks the partition,
the top walk and the exchange; the concatenated solution must match the
oracle's solve of the whole system to 1e-12 (the Err formula,
direct_solve.cc:216-225).  The same walk with the GPU bodies runs in
test_gpu_shard.py.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class OracleBodies:
    """The shard walk's task bodies on the CPU, from the oracle."""

    def __init__(self, R):
        import torch
        self.R, self.torch = R, torch

    def sub_solve(self, shape, Dg, Ug, Vg, Bg):
        R = self.R
        tree = R.build_tree(*shape)
        s = R.System(tree, Dg, Ug, Vg, Bg)
        X, _ = R.bfs_solve(s, nthreads=2)
        return np.asfortranarray(X[:, : shape[1]])

    def upload(self, a):
        return np.asfortranarray(a)

    def reduce(self, V, X, ncol):
        R = self.R
        k, r = V.shape
        W = np.zeros((r, ncol), order="F")
        V = np.asfortranarray(V)
        R.lib().ref_gemm_reduce(1.0, k, r, ncol, R._p(V), k, R._p(X), X.shape[0], 0, R._p(W), r)
        return W

    def node_solve(self, W0, W1, cw):
        R = self.R
        V0Td0, V0Tu0 = np.asfortranarray(W0[:, :cw]), np.asfortranarray(W0[:, cw:])
        V1Td1, V1Tu1 = np.asfortranarray(W1[:, :cw]), np.asfortranarray(W1[:, cw:])
        r1, r0 = V0Tu0.shape
        info = R.lib().ref_lu_node_solve(r0, r1, cw, R._p(V0Tu0), r1, R._p(V1Tu1), r0,
                                         R._p(V0Td0), r1, R._p(V1Td1), r0)
        assert info == 0
        return V1Td1, V0Td0

    def broadcast(self, X, u_col_beg, r, eta, ncol):
        R = self.R
        eta = np.asfortranarray(eta)
        R.lib().ref_gemm_broadcast(-1.0, 1.0, X.shape[0], r, ncol, R._p(X), X.shape[0],
                                   u_col_beg, R._p(eta), eta.shape[0], 0)

    def exchange_buffer(self, nslots, rows, cols):
        return self.torch.zeros((nslots, cols, rows), dtype=self.torch.float64)

    def to_exchange(self, W):
        return self.torch.from_numpy(np.ascontiguousarray(W))

    def from_exchange(self, t):
        return np.asfortranarray(t.numpy())

    def host(self, X):
        return np.asarray(X)


def _worker(rank, ws, port, shape, seed, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from oracle import refcpu as R
    from fastsolver_b200.shard import ShardedSolver, SubtreeSplit, TorchComm

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=120))
    try:
        N, m, r, t = shape
        s = R.gaussian_system(N, m, r, t, seed=seed)
        split = SubtreeSplit(N, m, r, t, ws, tree=s.tree)
        parts = split.local_arrays(rank, s.D, s.U, s.V, s.B)
        X = ShardedSolver(split, rank, TorchComm(), bodies=OracleBodies(R)).solve(*parts)
        out[rank] = (split.rows(rank), np.asarray(X))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,shape", [(2, (4096, 3, 16, 256)), (4, (5000, 2, 12, 300)),
                                      (2, (3001, 1, 10, 200))])
def test_sharded_solve_matches_oracle(oracle, ws, shape):
    seed = 77 + ws
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(ws, _free_port(), shape, seed, out), nprocs=ws,
                       join=True, start_method="spawn")
    N, m, r, t = shape
    s = oracle.gaussian_system(N, m, r, t, seed=seed)
    Xo, _ = oracle.bfs_solve(s, nthreads=4)
    X = np.zeros((N, m))
    covered = 0
    for g in range(ws):
        (rb, n), Xg = out[g]
        X[rb:rb + n] = Xg
        covered += n
    assert covered == N
    assert oracle.rel_error(X, Xo[:, :m]) < 1e-12
    assert oracle.relres(s, X) < 1e-13


def test_split_layout(fs, oracle):
    """The parts' sub-systems have the global subtree's shape (the sub-tree
    built from (N_g, m + r k, r, t) is the global subtree with column
    offsets shifted by r k), and their top paths reach the root."""
    from fastsolver_b200.shard import SubtreeSplit
    N, m, r, t = 262144, 16, 64, 512
    for P in (1, 2, 4, 8):
        sp = SubtreeSplit(N, m, r, t, P)
        assert sum(sp.rows(g)[1] for g in range(P)) == N
        for g in range(P):
            n, mg, _, _ = sp.sub_shape(g)
            sub = fs.build_tree(n, mg, r, t)
            glob = sp.tree
            # same number of nodes as the global subtree below the part's root
            below = [i for i in range(glob.shape[0])
                     if _under(glob, i, sp.roots[g])]
            assert sub.shape[0] == len(below)
            assert len(sp.ancestors(g)) == sp.k
    with pytest.raises(ValueError):
        SubtreeSplit(N, m, r, t, 3)


def _under(tree, i, root):
    while i != -1:
        if i == root:
            return True
        i = int(tree[i, 6])
    return False
