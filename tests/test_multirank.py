"""The N > 1 host path of bench.py on CPU: two gloo ranks (no GPU).

bench.py runs one independent replica per GPU (the path has no exchange
step), so its only collectives are the timing barrier and the max over
ranks; the job's throughput counts every rank's frames over the slowest
rank's time. These tests run those helpers as two real processes.
"""
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


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import torch
    import bench
    r, local, w, dist = bench.dist_setup(world, backend="gloo")
    assert (r, local, w) == (rank, rank, world)
    bench.barrier(dist, torch)
    slowest = bench.max_over_ranks(10.0 + 5.0 * rank, dist, torch)  # rank 1 is slower
    out[rank] = (slowest, bench.replica_work(100, w))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_time_is_the_slowest_and_work_adds_up():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    assert out[0] == out[1] == (15.0, 200)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import torch
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    r, local, w, dist = bench.dist_setup(1)
    assert (r, local, w, dist) == (0, 0, 1, None)
    assert bench.max_over_ranks(3.5, dist, torch) == 3.5


def _rank_leaves(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import torch
    import bench
    _, _, _, dist = bench.dist_setup(world, backend="gloo")
    bench.barrier(dist, torch)
    if rank == 1:
        os._exit(0)  # a rank that leaves between steps, none of its work in flight
    try:
        bench.max_over_ranks(1.0, dist, torch)
        out[rank] = "completed"
    except Exception as e:  # the survivor learns of it from its next collective
        out[rank] = "error: " + type(e).__name__


def test_a_rank_that_leaves_fails_the_next_collective():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    ctx = mp.start_processes(_rank_leaves, args=(world, port, out), nprocs=world, join=False,
                             start_method="spawn")
    for p in ctx.processes:
        p.join(timeout=150)
    assert out.get(0, "").startswith("error"), out.copy()
