"""The N > 1 (replica) path of bench.py on CPU: two gloo ranks exchange
their step times, both see the max, and the whole-job value counts every
rank's micrograph."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.reduce_max_over_ranks([100.0 + 50.0 * rank, 2.0 - rank], world, "cpu")
        dist.barrier()
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_value():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == [150.0, 2.0]
    import bench
    assert bench.replica_value(2, 150.0) == pytest.approx(2 * 1000.0 / 150.0)
    assert bench.reduce_max_over_ranks([3.0], 1) == [3.0]
