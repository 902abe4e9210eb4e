"""The multi-GPU paths of bench.py have no data-path collective: a single
scene runs as replicas, and the batched scenes are partitioned over the
ranks by particle count (every rank computes the same partition); the
whole-job figures are the slowest rank's time and the sum of the ranks'
particles.  Checked here with two and three gloo ranks on the CPU (the same
calls run over NCCL on GPUs)."""
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


def _batch_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine, counts = bench.batch_share(24, rank, world)
    units = sum(counts[i] for i in mine)
    ms, total = bench.job_reduce(5.0 + rank, units, world, device="cpu")
    out[rank] = (mine, units, ms, total, sum(counts), max(counts))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_batch_scenes_partitioned_over_gloo_ranks(world):
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_batch_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    seen = sorted(i for r in range(world) for i in out[r][0])
    n_all = out[0][4]
    assert seen == list(range(24))  # every scene on exactly one rank
    for r in range(world):
        assert out[r][3] == n_all  # the whole job's particles
        assert out[r][2] == 5.0 + (world - 1)  # the slowest rank's time
    loads = [out[r][1] for r in range(world)]
    assert max(loads) - min(loads) <= out[0][5]  # largest-first greedy bound


def test_partition_is_deterministic_and_balanced():
    sys.path.insert(0, str(ROOT))
    from exagoop_b200 import scenes
    counts = scenes.batched_scene_particle_counts()
    assert sum(counts) > 5e7 and len(counts) == 64
    for world in (1, 2, 4, 8):
        parts = scenes.partition_scenes(counts, world)
        assert parts == scenes.partition_scenes(counts, world)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(counts[i] for i in p) for p in parts]
        assert max(loads) <= sum(counts) / world + max(counts)
    # the counts are the lattice sizes the generator produces
    got = [p.n for _, p in scenes.batched_dam_breaks(n_scenes=5, seed=11, sides=(32, 48))]
    assert got == scenes.batched_scene_particle_counts(n_scenes=5, seed=11, sides=(32, 48))
