"""The multi-GPU path of bench.py is replicas: each rank advances its own
torus and the job's time is the slowest rank's.  The max-over-ranks
reduction and the whole-job value run here on two gloo ranks (CPU)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms_local = [12.5, 30.0][rank]
        ms_max = bench.replica_max(ms_local, dist, "cpu")
        out[rank] = (ms_max, bench.replica_value(4096, 10, world, ms_max))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1]
    ms_max, value = out[0]
    assert ms_max == 30.0
    assert value == pytest.approx(4096 * 10 * 2 / 0.030)
