"""The N > 1 bench path on CPU: world_size-2 gloo ranks.

Replicas share no data path; the only collectives are the barrier around the
timed region and the max over ranks of the elapsed time, so the whole job is
as slow as its slowest rank.  The reference arm runs on rank 0 alone.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        slowest = bench.max_over_ranks(world, 1.0 + rank)
        # The reference arm does no work off rank 0 (returns before sampling).
        ran = bench.run_reference(None, world, rank) if rank != 0 else None
        bench.barrier(world)
        out.put((rank, slowest, ran))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    results = sorted(out.get(timeout=5) for _ in range(2))
    assert [r[1] for r in results] == [2.0, 2.0]
    assert results[1][2] is None


def test_replica_value_is_aggregate_over_ranks():
    """value = world * steps / max-over-ranks seconds (weak scaling)."""
    import bench
    import inspect
    src = inspect.getsource(bench.run_b200)
    assert "value = world * args.steps / seconds" in src
    assert "max_over_ranks(world" in src


def test_reference_arm_ranks_join_no_process_group(monkeypatch):
    """Under torchrun the reference arm's ranks take no collective step, so
    they create no process group: rank 0 runs the reference's CPU solve
    alone and the other ranks exit at once, with nothing left to shut down."""
    import argparse
    import bench
    import torch.distributed as dist
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    world, rank, local = bench.dist_setup(argparse.Namespace(impl="reference"))
    assert (world, rank, local) == (2, 1, 1)
    assert not dist.is_initialized()
