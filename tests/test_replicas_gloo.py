"""Multi-rank host logic of bench.py on CPU: two ranks over gloo (127.0.0.1)
agree on the slowest rank's time and report the whole job's throughput as
the work of all replicas over that time.  The MD path itself runs replicas
only (one independent box per rank, no data-path collective)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 100.0 + 50.0 * rank                           # rank 1 is the slower one
    slow = bench.max_over_ranks(ms, dist, device="cpu")
    out[rank] = (slow, bench.job_rate(1000, world, slow / 1e3))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_max_time_and_summed_work():
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    slow, rate = res[0]
    assert slow == pytest.approx(150.0)
    assert rate == pytest.approx(2 * 1000 / 0.150)
