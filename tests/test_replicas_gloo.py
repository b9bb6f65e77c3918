"""Multi-process (world size 2, gloo, CPU) check of the replica aggregation
that bench.py uses under torchrun: each rank times its own solve, the job's
step time is the max over ranks, and the value counts every rank's solve."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, ms_per_rank, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.rank_max(ms_per_rank[rank], dist, "cpu")
        out[rank] = (ms, bench.replica_value(ms, ws))
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    ws = 2
    ms_per_rank = [30.0, 42.0]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(ws, _free_port(), ms_per_rank, out), nprocs=ws,
                       join=True, start_method="spawn")
    for r in range(ws):
        ms, v = out[r]
        assert ms == pytest.approx(42.0)
        assert v == pytest.approx(2 * 1e3 / 42.0)


def test_single_rank_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_max(12.5) == 12.5
    assert bench.replica_value(25.0, 1) == pytest.approx(40.0)
