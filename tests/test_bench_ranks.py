"""bench.py's multi-rank path: every rank reports its own time and the
line carries the maximum over ranks.  Two gloo ranks on CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r measured 10 * (r + 1) ms; all ranks must see the slowest
        got = bench.max_over_ranks(10.0 * (rank + 1), dist, torch.device("cpu"))
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ws = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(ws, port, out), nprocs=ws, join=True,
                           start_method="spawn")
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_max_over_ranks_single_process():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(3.5, None, None) == 3.5
