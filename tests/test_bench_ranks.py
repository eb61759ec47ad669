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


def test_whole_path_roofline_arithmetic():
    """bench.py's per-stage roofline: GEMM stages against the int8 figure, the rest against HBM,
    summed and set against the measured time per product (N=65536, L=1747, r=3636)."""
    bench = _bench()
    info = {"primes": 3636, "padded_primes": 3648, "words": 1752}
    stage_ms = {"pad": 0.31, "convert": 8.8, "forward": 2.0, "pointwise": 0.67, "inverse": 1.2,
                "transpose": 0.3, "crt": 4.4, "reduce": 0.6}
    out = bench.path_roofline(65536, 1747, info, stage_ms, 18.6, 2766.0, 6549.4)
    stages = out["stages"]
    assert stages["convert"]["bound"] == "int8 tensor" and stages["reduce"]["bound"] == "hbm"
    assert stages["convert"]["work"] == 2.0 * (2 * 65536) * (4 * 1747) * (4 * 3636)
    assert stages["forward"]["work"] == 4.0 * 2 * 2 * 3636 * 65536
    assert stages["convert"]["roof_ms"] == pytest.approx(stages["convert"]["work"] / 2766e12 * 1e3, abs=1e-4)
    assert stages["pointwise"]["roof_ms"] == pytest.approx(4.0 * 3 * 3636 * 65536 / 6549.4e9 * 1e3, abs=1e-4)
    assert out["roof_ms"] == pytest.approx(sum(s["roof_ms"] for s in stages.values()), abs=1e-2)
    assert out["measured_over_roof"] == pytest.approx(18.6 / out["roof_ms"], rel=1e-2)
    assert 16.0 < out["roof_ms"] < 17.0  # 14.4 ms of GEMMs + 2.1 ms of HBM stages
