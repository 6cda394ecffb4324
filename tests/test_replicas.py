"""Multi-GPU path of bench.py: one process per GPU, independent replicas (the
SIMP path does not shard; there is no data-path collective).  The only
cross-rank steps are the barrier around the timed region and the max over
ranks of the elapsed time; both run here on CPU with the gloo backend and two
ranks."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench.barrier(dist)
    t = bench.max_over_ranks(1.0 + rank, dist)  # rank r "took" 1 + r seconds
    out[rank] = (t, bench.job_rate(10, t, world))
    bench.barrier(dist)
    dist.destroy_process_group()


def test_replicas_report_the_slowest_rank_and_the_whole_job_rate():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0  # max over ranks
    assert res[0][1] == pytest.approx(world * 10 / 2.0)
