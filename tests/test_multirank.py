"""The multi-GPU path of bench.py is replicas with no data-path collective:
every rank times its own scene and the whole-job figures are the slowest
rank's time and the sum of the ranks' particles.  Checked here with two
gloo ranks on the CPU (the same calls run over NCCL on GPUs)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    ms, units = bench.job_reduce(10.0 * (rank + 1), 1000 * (rank + 1), world, device="cpu")
    out[rank] = (ms, units)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replica_reduction_over_gloo(world):
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        assert out[r] == (10.0 * world, 1000 * world * (world + 1) // 2)


def test_single_rank_reduction_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.job_reduce(3.5, 42, 1) == (3.5, 42)
