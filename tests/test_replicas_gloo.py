"""The N > 1 bench path ("replicas only"): two gloo ranks on the CPU run the
same max-over-ranks time reduction and whole-job value as bench.py."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [12.0, 15.5][rank]
        slowest = bench.max_over_ranks(ms, "cpu")
        dist.barrier()
        out[rank] = (slowest, bench.whole_job_value(world, 1000, 10, slowest))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    slowest, value = res[0]
    assert slowest == 15.5
    assert abs(value - 2 * 1000 * 10 / 15.5e-3) < 1e-6 * value
