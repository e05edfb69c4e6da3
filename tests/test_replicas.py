"""The multi-GPU form of bench.py is N independent replicas: each rank times its own solve,
the job's time is the slowest rank's (max over ranks), and the job's rate counts every rank's
work.  Checked here with two gloo ranks on the CPU (no GPU needed)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


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
    local_ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
    slowest = bench.max_over_ranks(dist, local_ms, "cpu")
    out[rank] = (slowest, bench.replicas_value(2.0e12, world, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_two_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        slowest, rate = res[rank]
        assert slowest == 15.0
        assert abs(rate - 2.0e12 * 2 / 15e-3) < 1.0


def test_single_rank_is_plain():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.max_over_ranks(None, 7.5, "cpu") == 7.5
    assert bench.replicas_value(1.0e12, 1, 10.0) == 1.0e14
