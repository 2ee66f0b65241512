"""bench.py's multi-GPU path is replicas (weak scaling, no data-path
collective): each rank advances its own grid, and rank 0 reports the
cell-updates of all ranks over the slowest rank's time.  Here two gloo ranks
on the CPU exercise that reduction with rank-specific numbers."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: (r+1) * 1e9 updates in (r+1) * 100 ms
        rate, ms_max, total = bench.whole_job_rate((rank + 1) * 1e9, (rank + 1) * 100.0, world,
                                                   "cpu")
        out[rank] = (rate, ms_max, total)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replica_reduction_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        rate, ms_max, total = res[r]
        assert ms_max == 200.0
        assert total == 3e9
        assert rate == pytest.approx(3e9 / 0.2)
