"""Replica timing of bench.py on two host-only ranks (gloo): every rank reports its own step time, the line carries
the maximum, the barrier releases both ranks, and the reference arm does its work on rank 0 only."""
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
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    import bench

    value = bench.max_over_ranks(1.5 + rank, world)
    bench.barrier(world)
    args = type("Args", (), {})()
    skipped = bench.bench_reference(args, rank, world, rank) if rank != 0 else None
    out.put((rank, value, skipped))
    dist.destroy_process_group()


def test_max_over_ranks_and_barrier_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r for r, _, _ in results) == [0, 1]
    assert all(v == pytest.approx(2.5) for _, v, _ in results)
    assert all(s is None for _, _, s in results)


def test_solver_launch_count_formula():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.mg_grid_levels(128) == (8, 4)   # 128 64 32 16 on the grid, 8 4 2 1 in one block
    assert bench.mg_grid_levels(12) == (5, 1)    # 12 on the grid, 6 3 2 1 in one block
    # per iteration: 3 coarse grid levels x (restrict, prolong + smooth) + block + prolong0 + smooth0 + p/q + update
    assert bench.solver_launches(128, 15, 3) == 2 + 3 * 4 + 11 * 15
    # 256^3: level 1 (128^3) keeps prolongation and smoothing apart, levels 2-4 fuse them
    assert bench.mg_grid_levels(256) == (9, 5)
    assert bench.solver_launches(256, 12, 1) == 2 + 3 * 2 + (3 + 2 + 2 + 2 + 5) * 12
