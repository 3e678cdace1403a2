"""Replica ranks of bench.py on CPU (gloo, world size 2): whole-job value is
all ranks' units over the slowest rank's time; the reference arm runs on
rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks(backend="gloo")
    units, secs, value = bench.combine(r, 100.0 * (rank + 1), 2.0 + rank)
    r.barrier()
    r.close()
    q.put((rank, units, secs, value))


def test_combine_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, units, secs, value in res:
        assert units == 300.0 and secs == 3.0 and value == pytest.approx(100.0)


def test_single_rank_combine():
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks()
    assert bench.combine(r, 50.0, 2.0) == (50.0, 2.0, 25.0)
