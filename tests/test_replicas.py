"""The multi-GPU path of bench.py is replicas: each rank steps its own copy
(or its share of an ensemble's runs) with no collective while stepping, and
the reported figures combine the ranks' results (slowest rank's time, all
ranks' work). These host-side pieces run here as two gloo ranks on CPU."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, REPO)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, steps = bench.aggregate_over_ranks(10.0 + 5.0 * rank, 100 * (rank + 1))
        runs = bench.split_runs(list(range(11)), rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, runs)
        q.put((rank, ms, steps, gathered))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_aggregation_two_gloo_ranks():
    world, port = 2, 29517 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, steps, gathered in out:
        assert ms == 15.0 and steps == 300  # slowest rank's time, every rank's work
        flat = sorted(x for part in gathered for x in part)
        assert flat == list(range(11))  # every run on exactly one rank
        assert all(len(part) in (5, 6) for part in gathered)


def test_single_process_aggregation_is_local():
    sys.path.insert(0, REPO)
    import bench

    assert not dist.is_initialized()
    assert bench.aggregate_over_ranks(7.5, 42) == (7.5, 42)
    assert bench.split_runs("abcde", 0, 1) == list("abcde")


def test_ensemble_smaller_than_world_is_rejected():
    """An ensemble with fewer runs than ranks would leave a rank without work
    while its peers wait for it in the aggregation: bench.py refuses it."""
    import subprocess

    env = dict(os.environ, WORLD_SIZE="4", RANK="0", LOCAL_RANK="0")
    res = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--ensemble", "3"], env=env,
                         capture_output=True, text=True, timeout=120)
    assert res.returncode == 2
    assert "smaller than the number of ranks" in res.stderr
