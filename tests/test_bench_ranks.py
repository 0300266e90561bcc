"""bench.py's multi-GPU timing rule on CPU: with N replicas (one process per
GPU, no data-path collective), the job's time is the maximum over ranks of
each rank's own device time.  Two gloo ranks on 127.0.0.1 stand in for two
GPUs."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(torch, values[rank], torch.device("cpu"), world)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("values", [(0.125, 0.25), (3.0, 1.0)])
def test_max_over_ranks_gloo(values):
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, _free_port(), values, out), nprocs=world, join=True,
                           start_method="spawn")
        assert out[0] == out[1] == max(values)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, 0.5, torch.device("cpu"), 1) == 0.5
