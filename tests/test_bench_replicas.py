"""bench.py's multi-GPU plumbing on CPU: world size 2 over gloo.  The path shards as
independent replicas (one mesh per GPU, no collective on the data path); the only
collectives are the barrier around the timed region and the max over ranks of the time."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as td
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bench.barrier(td)
    ms = 10.0 + 5.0 * rank                  # the slower rank sets the job time
    ms_max = bench.allmax(td, ms)
    out[rank] = (ms_max, bench.aggregate(1000.0, world, ms_max))
    bench.barrier(td)
    td.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms_max, value = res[0]
    assert ms_max == 15.0
    assert value == pytest.approx(1000.0 * 2 / 0.015)
