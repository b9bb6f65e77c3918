"""The sharded solve with the GPU task bodies (fastsolver_b200.shard).

Two processes, one part each, share cuda:0 and exchange the top-level
partial reduces through gloo (host memory): no kernel of one process waits
on the other's, so sharing one GPU is safe.  Each part's sub-solve is the
library's fused FP64 solve of its subtree; the top levels run the C ABI's
reduce, LUSolve and broadcast bodies.  The concatenated solution must match
the oracle's solve of the whole system to 1e-12.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, shape, seed, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from oracle import refcpu as R
    from fastsolver_b200.shard import ShardedSolver, SubtreeSplit, TorchComm

    torch.cuda.set_device(0)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=120))
    try:
        N, m, r, t = shape
        s = R.gaussian_system(N, m, r, t, seed=seed)
        split = SubtreeSplit(N, m, r, t, ws)
        parts = split.local_arrays(rank, s.D, s.U, s.V, s.B)
        X = ShardedSolver(split, rank, TorchComm()).solve(*parts)
        out[rank] = (split.rows(rank), np.asarray(X))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,shape", [(2, (16384, 4, 32, 512)), (2, (3001, 2, 10, 200))])
def test_gpu_sharded_solve_matches_oracle(oracle, cuda, ws, shape):
    seed = 91
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(ws, _free_port(), shape, seed, out), nprocs=ws,
                       join=True, start_method="spawn")
    N, m, r, t = shape
    s = oracle.gaussian_system(N, m, r, t, seed=seed)
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    X = np.zeros((N, m))
    for g in range(ws):
        (rb, n), Xg = out[g]
        X[rb:rb + n] = Xg
    assert oracle.rel_error(X, Xo[:, :m]) < 1e-12
    assert oracle.relres(s, X) < 1e-13
