"""The replicas-only multi-GPU path of bench.py on CPU ranks (gloo,
world_size 2): the max-over-ranks timing reduction, the whole-job rate, the
per-rank seeds, and the reference arm running on rank 0 only."""

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


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank                      # rank 1 is the slower replica
        got = bench.max_over_ranks(ms, "cpu", world)
        rate = bench.replica_rate(world, 3, got)
        args = type("A", (), {"config": "c1", "warmup": 0, "steps": 1})()
        ref = bench.run_reference(args, rank, world) if rank != 0 else "skipped"
        q.put((rank, got, rate, ref, bench.SEED + rank))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [150.0, 150.0]           # both ranks see the slower one
    assert res[0][2] == pytest.approx(2 * 3 / 0.150)        # whole-job sweeps/s
    assert res[1][3] is None                                 # the reference arm: rank 0 only
    assert res[0][4] != res[1][4]                            # independent replica seeds


def test_single_rank_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, "cpu", 1) == 12.5
    assert bench.replica_rate(1, 4, 2000.0) == pytest.approx(2.0)
