"""The replicas-only multi-GPU path of bench.py (independent instances per
rank, no data-path collective): its aggregation over ranks -- the slowest
rank's time and the sum of the ranks' particles -- checked with two gloo
ranks on the CPU, as torchrun would launch them on one node."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [10.0, 25.0][rank]            # rank 1 is the slow one
    n = [1000, 3000][rank]
    out[rank] = (bench.dist_max(ms, world), bench.dist_sum(n, world), bench.replica_value(n, 4, ms, world))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_two_gloo_ranks():
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    for r in range(2):
        mx, total, value = out[r]
        assert mx == 25.0 and total == 4000.0
        assert value == pytest.approx(4000.0 * 4 / 0.025)
