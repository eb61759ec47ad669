"""Batched and serving forms through the C ABI: bit-exact per instance, alone and in the mix."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cudart():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.init()
    lib = ctypes.CDLL("libcudart.so.12")
    lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    lib.cudaDeviceSynchronize.argtypes = []
    return lib


H2D, D2H = 1, 2


def uneven_points(inputs, count, seed, sizes=(256, 512, 1024, 2048, 4096), limb_range=(1, 160)):
    rng = np.random.Generator(np.random.PCG64(seed))
    points = []
    for i in range(count):
        n = int(rng.choice(sizes))
        limbs = int(np.exp(rng.uniform(np.log(limb_range[0]), np.log(limb_range[1]))))
        q, a, b = inputs.instance(n, limbs, seed * 1000 + i, 0)
        points.append((n, limbs, q, a, b))
    return points


def test_batch_graph_matches_oracle_and_plain_path(fpc, inputs, oracle, cudart):
    points = uneven_points(inputs, 12, 7)
    with fpc.Batch([(n, 32 * l, l, q) for n, l, q, _, _ in points], lanes=3) as batch:
        for i, (n, l, q, a, b) in enumerate(points):
            da, db, dc = batch.io(i)
            assert cudart.cudaMemcpy(da, a.ctypes.data, a.nbytes, H2D) == 0
            assert cudart.cudaMemcpy(db, b.ctypes.data, b.nbytes, H2D) == 0
        for _ in range(2):  # the graph can be relaunched
            batch.run_device(0)
            assert cudart.cudaDeviceSynchronize() == 0
            for i, (n, l, q, a, b) in enumerate(points):
                c = np.empty_like(a)
                assert cudart.cudaMemcpy(c.ctypes.data, batch.io(i)[2], c.nbytes, D2H) == 0
                assert np.array_equal(c, oracle.kronecker(q, a, b)), (i, n, l)
        # the plain per-call path over the same plans gives the same products
        for i, (n, l, q, a, b) in enumerate(points):
            batch.run_one(i, 0)
            assert cudart.cudaDeviceSynchronize() == 0
            c = np.empty_like(a)
            assert cudart.cudaMemcpy(c.ctypes.data, batch.io(i)[2], c.nbytes, D2H) == 0
            assert np.array_equal(c, oracle.kronecker(q, a, b)), i
        lanes = {batch.info(i)["lane"] for i in range(len(points))}
        assert lanes == {0, 1, 2}


def test_batch_single_lane_pipeline(fpc, inputs, oracle):
    """One compute lane (CTA-pair GEMMs) with copy-in / copy-out streams, host arrays in and out."""
    points = uneven_points(inputs, 8, 13, sizes=(1024, 4096, 8192), limb_range=(16, 300))
    with fpc.Batch([(n, 32 * l, l, q) for n, l, q, _, _ in points], lanes=1) as batch:
        assert {batch.info(i)["lane"] for i in range(len(points))} == {0}
        for _ in range(2):
            results = batch.run([p[3] for p in points], [p[4] for p in points])
            for (n, l, q, a, b), c in zip(points, results):
                assert np.array_equal(c, oracle.kronecker(q, a, b)), (n, l)


def test_batch_two_phases_by_default(fpc, inputs, oracle, cudart):
    """Default lanes: small instances share the GPU on several lanes (single-CTA GEMMs), then the
    large one runs alone on lane 0 with CTA-pair GEMMs; device graph and host arrays both exact."""
    points = uneven_points(inputs, 9, 17, sizes=(1024, 2048, 4096), limb_range=(8, 90))
    q, a, b = inputs.instance(65536, 300, 1717, 0)  # estimated at well over 1 ms: the sequential phase
    points.append((65536, 300, q, a, b))
    with fpc.Batch([(n, 32 * l, l, q) for n, l, q, _, _ in points]) as batch:
        lanes = [batch.info(i)["lane"] for i in range(len(points))]
        assert len(set(lanes[:-1])) > 1 and lanes[-1] == 0, lanes
        assert batch.info(len(points) - 1)["gemm"] == 3
        want = [oracle.kronecker(q, a, b) for _, _, q, a, b in points]
        for i, (n, l, q, a, b) in enumerate(points):
            da, db, _ = batch.io(i)
            assert cudart.cudaMemcpy(da, a.ctypes.data, a.nbytes, H2D) == 0
            assert cudart.cudaMemcpy(db, b.ctypes.data, b.nbytes, H2D) == 0
        batch.run_device(0)
        assert not batch.status().any()
        for i, (n, l, q, a, b) in enumerate(points):
            c = np.empty_like(a)
            assert cudart.cudaMemcpy(c.ctypes.data, batch.io(i)[2], c.nbytes, D2H) == 0
            assert np.array_equal(c, want[i]), (i, n, l)
        results = batch.run([p[3] for p in points], [p[4] for p in points])
        for i, c in enumerate(results):
            assert np.array_equal(c, want[i]), i


def test_batch_host_path_and_autotuner(fpc, inputs, oracle, tmp_path):
    points = uneven_points(inputs, 6, 11, sizes=(1024, 4096), limb_range=(29, 80))
    cache = str(tmp_path / "tune.txt")
    specs = [(n, 32 * l, l, q) for n, l, q, _, _ in points]
    with fpc.Batch(specs, lanes=2, tune=True, tune_cache=cache) as batch:
        results = batch.run([p[3] for p in points], [p[4] for p in points])
        for (n, l, q, a, b), c in zip(points, results):
            assert np.array_equal(c, oracle.kronecker(q, a, b))
        tuned = [batch.info(i) for i in range(len(points))]
    assert all(t["tuned_ms"] > 0 for t in tuned)
    lines = [x for x in open(cache).read().splitlines() if not x.startswith("#")]
    assert len(lines) == len({(n, l) for n, l, *_ in points})
    # a second batch reads the cache instead of tuning again
    with fpc.Batch(specs, lanes=2, tune=True, tune_cache=cache) as batch:
        again = [batch.info(i)["tuned_ms"] for i in range(len(points))]
    assert again == pytest.approx([t["tuned_ms"] for t in tuned], rel=1e-9)


def test_server_results_alone_equal_results_in_the_mix(fpc, inputs, oracle):
    limbs = 64
    q = inputs.random_modulus(limbs, 200)
    rng = np.random.Generator(np.random.PCG64(5))
    requests = []
    for i in range(24):
        n = int(rng.choice([1024, 2048, 4096]))
        requests.append((inputs.random_operand(rng, n, q), inputs.random_operand(rng, n, q)))
    with fpc.Server(slots=4, hbm_budget=8 << 30) as server:
        session = server.open_session(32 * limbs, limbs, q, ns=[1024, 2048, 4096])
        alone = []
        for a, b in requests[:4]:  # one at a time
            c, latency = server.wait(server.submit(session, a, b))
            alone.append(c)
        ids = [server.submit(session, a, b) for a, b in requests]  # all at once: they overlap
        mixed = [server.wait(rid)[0] for rid in ids]
        stats = server.stats()
    for i in range(4):
        assert np.array_equal(alone[i], mixed[i])
    for (a, b), c in zip(requests, mixed):
        assert np.array_equal(c, oracle.kronecker(q, a, b))
    assert stats["completed"] == 28 and stats["failed"] == 0
    assert 0 < stats["p50_ms"] <= stats["p99_ms"]


def test_server_admission_respects_the_budget(fpc, inputs):
    limbs = 32
    q = inputs.random_modulus(limbs, 201)
    with fpc.Server(slots=2, hbm_budget=64 << 20) as server:  # plan tables fit, a large request does not
        session = server.open_session(32 * limbs, limbs, q, ns=[256])
        a = np.zeros((256, limbs), np.uint32)
        c, _ = server.wait(server.submit(session, a, a))
        assert not c.any()
        big = np.zeros((65536, limbs), np.uint32)
        with pytest.raises(RuntimeError, match="budget"):
            server.wait(server.submit(session, big, big))
        assert server.stats()["failed"] == 1


def test_server_refuses_beyond_its_queue_bound(fpc, inputs):
    """Under overload the serving form sheds load at submit (NEGACYCLIC_EBUSY) instead of letting
    its queue grow: with one slot and a queue bound of two, a burst is partly refused, the rest
    completes, and the stats count both and the deepest queue seen."""
    limbs = 64
    q = inputs.random_modulus(limbs, 202)
    rng = np.random.Generator(np.random.PCG64(9))
    a = inputs.random_operand(rng, 65536, q)
    b = inputs.random_operand(rng, 65536, q)
    with fpc.Server(slots=1, max_queue=2, hbm_budget=8 << 30) as server:
        session = server.open_session(32 * limbs, limbs, q, ns=[65536])
        first, _ = server.wait(server.submit(session, a, b))  # warm
        ids = [server.submit(session, a, b) for _ in range(24)]
        accepted = [rid for rid in ids if rid is not None]
        assert 0 < len(accepted) < len(ids)
        for rid in accepted:
            c, _ = server.wait(rid)
            assert np.array_equal(c, first)
        stats = server.stats()
    assert stats["rejected"] == len(ids) - len(accepted)
    assert stats["completed"] == 1 + len(accepted) and stats["failed"] == 0
    assert 1 <= stats["max_queued"] <= 2
