"""The multi-process side of bench.py, on CPU: two gloo ranks, launched the way
torchrun launches bench.py on two GPUs (RANK / WORLD_SIZE / MASTER_* in the
environment, 127.0.0.1 rendezvous).

Multi-GPU here is replicas only: each rank runs its own product stream, the only
collectives are the barrier and one all-reduce (MAX) of a scalar time, and the
whole-job value is world * steps / slowest time. The reference arm runs on rank 0
alone; other ranks return at once without work or output.
"""
import contextlib
import importlib.util
import io
import os
import socket
import sys
import types

import pytest

from conftest import REPO


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(REPO, "bench.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def _rank_main(rank: int, world: int, port: int, results):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        assert bench.distributed() == (world, rank, rank)
        # each replica reports its own time; every rank must see the slowest
        own = 1.0 + 0.25 * rank
        slowest = bench.max_over_ranks(own, world)
        value = bench.replica_throughput(world, 10, slowest)
        dist.barrier()
        # reference arm: rank 0 alone works and prints; the others return at once
        printed = io.StringIO()
        if rank != 0:
            with contextlib.redirect_stdout(printed):
                bench.run_reference(types.SimpleNamespace(steps=1, warmup=0))
        results.put((rank, own, slowest, value, printed.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    results = ctx.SimpleQueue()
    mp.start_processes(_rank_main, args=(world, port, results), nprocs=world, join=True, start_method="spawn")
    rows = sorted(results.get() for _ in range(world))
    slowest = max(own for _, own, _, _, _ in rows)
    for rank, own, seen, value, printed in rows:
        assert seen == slowest
        assert value == pytest.approx(world * 10 / slowest)
        if rank != 0:
            assert printed == ""


def test_single_process_needs_no_process_group():
    bench = _bench()
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_throughput(1, 20, 0.5) == 40.0
