"""Parity of the CUDA path (through the C ABI) with the reference checker and the oracle.

Bit-exact everywhere: the product is integer arithmetic, the tolerance is 0.
"""
import json
import os

import numpy as np
import pytest

import cases
import model
from test_oracle import baseline_points, edge_pair, point_pairs, reference_points, as_array

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    return t


# ---------------------------------------------------------------- raw byte GEMM

@pytest.mark.parametrize("m,n,k", [(128, 256, 128), (300, 520, 400), (1024, 768, 2048), (256, 512, 33024),
                                   (4096, 1280, 1024)])
def test_tensor_gemm_matches_simt_and_numpy(m, n, k, fpc, torch):
    gen = torch.Generator(device="cuda").manual_seed(m + n + k)
    a = torch.randint(0, 256, (m, k), dtype=torch.uint8, device="cuda", generator=gen)
    b = torch.randint(0, 256, (n, k), dtype=torch.uint8, device="cuda", generator=gen)
    if k == 33024:  # the int32 accumulation bound: all-255 rows
        a[0].fill_(255)
        b[0].fill_(255)
    outs = {}
    lib = fpc.library()
    for engine in (fpc.GEMM_SIMT, fpc.GEMM_TENSOR, fpc.GEMM_TENSOR_SINGLE):
        d = torch.full((m, n), -1, dtype=torch.int32, device="cuda")
        status = lib.negacyclic_gemm_u8(a.data_ptr(), b.data_ptr(), d.data_ptr(), m, n, k, engine, None)
        assert status == 0, fpc.last_error()
        torch.cuda.synchronize()
        outs[engine] = d.cpu().numpy()
    want = a.cpu().numpy().astype(np.int64) @ b.cpu().numpy().astype(np.int64).T
    assert np.array_equal(outs[fpc.GEMM_SIMT].astype(np.int64), want)
    assert np.array_equal(outs[fpc.GEMM_TENSOR].astype(np.int64), want)  # CTA-pair kernel
    assert np.array_equal(outs[fpc.GEMM_TENSOR_SINGLE].astype(np.int64), want)


# ---------------------------------------------------------------- reference checker points

ENGINES = {"auto": 0, "simt": 1}


@pytest.mark.parametrize("engine", sorted(ENGINES))
@pytest.mark.parametrize("point", reference_points(), ids=lambda p: f"N{p['N']}_W{p['W']}_{p['kind']}")
def test_reference_points_bit_exact(point, engine, fpc, inputs):
    q, pairs = point_pairs(point)
    limbs = point["L"]
    q_arr = inputs.from_int(q, limbs)
    with fpc.Plan(point["N"], point["W"], limbs, q_arr, gemm=ENGINES[engine]) as plan:
        for (a, b), expect in zip(pairs, point["cases"]):
            c = plan.run(as_array(a, limbs), as_array(b, limbs))
            assert cases.sha256(c.tobytes()) == expect["c_sha256"]


def test_plugin_interface_mirror(fpc, inputs):
    """fherma_init / fherma_run / fherma_free as the reference's harness calls them."""
    point = reference_points()[7]  # N=1024, W=512
    q, pairs = point_pairs(point)
    limbs = point["L"]
    state = fpc.fherma_init(fpc.Point(point["N"], point["W"], limbs, inputs.from_int(q, limbs)))
    try:
        for (a, b), expect in zip(pairs, point["cases"]):
            out = fpc.fherma_run(state, fpc.Inputs(as_array(a, limbs), as_array(b, limbs)))
            assert out.c.shape == (point["N"], limbs)
            assert cases.sha256(out.c.tobytes()) == expect["c_sha256"]
        with pytest.raises(RuntimeError, match="wrong input size"):
            fpc.fherma_run(state, fpc.Inputs(np.zeros((3, limbs), np.uint32), np.zeros((3, limbs), np.uint32)))
    finally:
        fpc.fherma_free(state)


# ---------------------------------------------------------------- random odd q (the benchmark's kind of modulus)

def baseline_cases(point, inputs):
    """(label, q, a, b, entry) of every hashed case of a point; operands are made one case at a
    time (full-size operands are 458 MB each)."""
    n, limbs, seed = point["N"], point["L"], point["seed"]
    q = inputs.random_modulus(limbs, seed)
    assert hex(inputs.to_int(q)) == point["q_hex"]
    for entry in point["cases"]:
        label = entry["label"]
        if label.startswith("seed"):
            _, a, b = inputs.instance(n, limbs, int(label[4:].split("_")[0]), int(label.split("index")[1]))
        else:
            x, y = edge_pair(inputs, label)
            a, b = inputs.edge_operand(n, q, x), inputs.edge_operand(n, q, y)
        yield label, q, a, b, entry


@pytest.mark.parametrize("point", [p for p in baseline_points() if p["N"] * p["L"] <= 4096 * 64],
                         ids=lambda p: f"N{p['N']}_L{p['L']}")
@pytest.mark.parametrize("engine", sorted(ENGINES))
def test_random_modulus_config_bit_exact(point, engine, fpc, inputs):
    plan = None
    for label, q, a, b, entry in baseline_cases(point, inputs):
        if plan is None:
            plan = fpc.Plan(point["N"], 32 * point["L"], point["L"], q, gemm=ENGINES[engine])
        c = plan.run(a, b)
        assert cases.sha256(c.tobytes()) == entry["c_sha256"], label
    plan.close()


@pytest.mark.parametrize("n,limbs,split", [(1, 1, 0), (2, 3, 0), (8, 2, 2), (64, 1, 0), (128, 29, 0),
                                           (256, 40, 2), (512, 33, 4), (2048, 17, 0), (4096, 70, 0),
                                           (8192, 32, 0), (16384, 9, 0), (1024, 1747, 0), (256, 3000, 0)])
def test_random_points_against_oracle(n, limbs, split, fpc, inputs, oracle):
    for index in range(2):
        q, a, b = inputs.instance(n, limbs, 1000 + n + limbs, index)
        want = oracle.kronecker(q, a, b)
        for engine in (0, 1):
            with fpc.Plan(n, 32 * limbs, limbs, q, split=split, gemm=engine) as plan:
                got = plan.run(a, b)
            assert np.array_equal(got, want), (n, limbs, split, engine, index)


@pytest.mark.parametrize("limbs", [3, 40])
def test_every_ring_split(limbs, fpc, inputs, oracle):
    """Ring splits 1 to 16 at N=8192 (transforms of 8192 down to 512 points, pointwise combines
    of 1 to 16 transforms): each gives the oracle's product."""
    n = 8192
    q, a, b = inputs.instance(n, limbs, 4242, 0)
    want = oracle.kronecker(q, a, b)
    for split in (1, 2, 4, 8, 16):
        with fpc.Plan(n, 32 * limbs, limbs, q, split=split) as plan:
            assert plan.info()["split"] == split
            assert np.array_equal(plan.run(a, b), want), split


def test_small_moduli(fpc, inputs, oracle):
    """q of one or two limbs, including q below a prime and q = 2, 3."""
    rng = np.random.Generator(np.random.PCG64(3))
    for qv in (2, 3, 5, 65537, 0xFFFFFFFF, (1 << 31) - 1, (1 << 61) - 1, (1 << 64) - 59):
        limbs = 1 if qv < (1 << 32) else 2
        q = inputs.from_int(qv, limbs)
        a = inputs.random_operand(rng, 512, q)
        b = inputs.random_operand(rng, 512, q)
        with fpc.Plan(512, 32 * limbs, limbs, q) as plan:
            assert np.array_equal(plan.run(a, b), oracle.kronecker(q, a, b)), qv


# ---------------------------------------------------------------- stage-by-stage against the model

@pytest.mark.parametrize("n,limbs,split", [(256, 4, 2), (512, 33, 1), (1024, 2, 4)])
def test_stages_match_model(n, limbs, split, fpc, inputs):
    q, a, b = inputs.instance(n, limbs, 77, 0)
    qi = inputs.to_int(q)
    ref = model.stages(model.make_plan(n, limbs, qi, split), inputs.poly_to_ints(a), inputs.poly_to_ints(b))
    with fpc.Plan(n, 32 * limbs, limbs, q, split=split) as plan:
        info = plan.info()
        c = plan.run(a, b)
        crt_in = np.frombuffer(plan.debug_read(1), np.uint32).reshape(n, info["padded_primes"])
        dots = np.frombuffer(plan.debug_read(2), np.uint64).reshape(n, info["words"])
    r = info["primes"]
    v = np.array(ref["v"], dtype=np.uint32).T  # [n][r]
    assert np.array_equal(crt_in[:, :r], v)
    assert not crt_in[:, r:].any()
    assert np.array_equal(dots, np.array(ref["dots"], dtype=np.uint64))
    assert inputs.poly_to_ints(c) == ref["c"]


# ---------------------------------------------------------------- device-resident entry point

def test_run_device_matches_run(fpc, inputs, torch):
    n, limbs = 4096, 64
    q, a, b = inputs.instance(n, limbs, 0, 0)
    with fpc.Plan(n, 32 * limbs, limbs, q) as plan:
        host = plan.run(a, b)
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(b.view(np.int32)).cuda()
        dc = torch.empty_like(da)
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):  # twice: internal buffers are reused
            plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream)
            torch.cuda.synchronize()
            assert np.array_equal(dc.cpu().numpy().view(np.uint32), host)


@pytest.mark.parametrize("limbs", [300, 100])  # 1200-byte rows: transform-ordered input; 400-byte: by coefficient
def test_streamed_host_path_with_sixteen_transforms(limbs, fpc, inputs, oracle, torch):
    """s = 16 gives 16 input chunks (the event budget) and the plain output split; the host path
    must equal the unchunked device path, and spot coefficients the schoolbook sums."""
    n = 65536
    q, a, b = inputs.instance(n, limbs, 31, 0)
    with fpc.Plan(n, 32 * limbs, limbs, q, split=16) as plan:
        assert plan.info()["split"] == 16
        host = plan.run(a, b)
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(b.view(np.int32)).cuda()
        dc = torch.empty_like(da)
        plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(dc.cpu().numpy().view(np.uint32), host)
    for i in (0, 1, 15, 16, 4097, n - 1):
        assert np.array_equal(oracle.schoolbook_at(q, a, b, i)[0], host[i]), i


@pytest.mark.parametrize("n,limbs", [(65536, 55), (32768, 28), (8192, 300)])
def test_host_path_locking_combinations(n, limbs, fpc, inputs, torch):
    """The host path with page-locked and pageable arrays in every combination: pageable inputs
    are packed by the host team (transform order when the ring is split), page-locked ones go
    straight to the copy engine (coefficient order for rows under 1 KB); pageable outputs are
    unpacked by the team as chunks land. All must equal the device-resident product."""
    q, a, b = inputs.instance(n, limbs, 4242, 0)
    with fpc.Plan(n, 32 * limbs, limbs, q) as plan:
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(b.view(np.int32)).cuda()
        dc = torch.empty_like(da)
        plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        want = dc.cpu().numpy().view(np.uint32)
        pin = lambda x: torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)  # noqa: E731
        pa, pb, pc = pin(a), pin(b), pin(np.zeros_like(a))
        for x, y, out in [(a, b, None), (pa, pb, pc), (pa, b, None), (a, pb, pc), (pa, pb, None), (a, b, pc)]:
            got = plan.run(x, y, out=out if out is not None else np.zeros_like(a))
            assert np.array_equal(got, want)
            if out is not None:
                out[:] = 0
        assert plan.status() == 0


# ---------------------------------------------------------------- full-size configurations

def big_points():
    return [p for p in baseline_points() if p["N"] * p["L"] > 4096 * 64]


def big_configs():
    """Full-size hashed points grouped by configuration (N, L): config 2 is one q (seed 1) with
    20 instances and every edge pair; config 3 is one q per seed 2..21, edge pairs with seed 2's."""
    groups = {}
    for p in big_points():
        groups.setdefault((p["N"], p["L"]), []).append(p)
    return [groups[key] for key in sorted(groups)]


def first_points():
    return [ps[0] for ps in big_configs()]


def _constant(x):
    """The common value of a polynomial whose coefficients are all equal, else None."""
    return int.from_bytes(x[0].astype("<u4").tobytes(), "little") if (x == x[0]).all() else None


@pytest.mark.parametrize("point", first_points(), ids=lambda p: f"N{p['N']}_L{p['L']}")
def test_full_size_edge_inputs(point, fpc, inputs, oracle):
    """Every edge pair of the reference's checks (zero, unit, all q-1, impulses at 0 and N-1,
    alternating q-1/q-2, 0xFFFFFFFF limbs below q, limb boundaries, q/2) at N=32768/L=868 and
    N=65536/L=1747, checked exactly without a full GMP product:
      constant a, b:       c_i = a b (2i + 2 - N) mod q (negacyclic sum of N equal terms)
      impulses:            one nonzero coefficient, at the shifted index
      q-1 at odd j, ones:  c_i = (q-1) (2 floor((i+1)/2) - N/2) mod q
      others:              direct coefficient sums (schoolbook) at spot indices."""
    n, limbs, seed = point["N"], point["L"], point["seed"]
    q = inputs.random_modulus(limbs, seed)
    qi = inputs.to_int(q)
    edges = inputs.edge_operands(n, q)
    with fpc.Plan(n, 32 * limbs, limbs, q) as plan:
        for x, y in inputs.EDGE_PAIRS:
            a, b = edges[x], edges[y]
            c = plan.run(a, b)
            got = inputs.poly_to_ints(c)
            ca, cb = _constant(a), _constant(b)
            if ca is not None and cb is not None:
                base = ca * cb % qi
                want = [base * (2 * i + 2 - n) % qi for i in range(n)]
            elif (x, y) == ("impulse0", "impulse_last"):  # 1 * (q-1) X^(N-1)
                want = [0] * n
                want[n - 1] = qi - 1
            elif (x, y) == ("impulse_last", "impulse_last"):  # (q-1)^2 X^(2N-2) = -X^(N-2)
                want = [0] * n
                want[n - 2] = qi - 1
            elif (x, y) == ("alt_zero", "ones"):
                want = [(qi - 1) * (2 * ((i + 1) // 2) - n // 2) % qi for i in range(n)]
            else:
                for i in (0, n // 2 + 1, n - 1):
                    assert np.array_equal(oracle.schoolbook_at(q, a, b, i)[0], c[i]), (x, y, i)
                continue
            assert got == want, (x, y)


@pytest.mark.parametrize("point", first_points(), ids=lambda p: f"N{p['N']}_L{p['L']}")
def test_full_size_seeded_instances(point, fpc, inputs, oracle):
    """Further seeded instances of the full-size configurations, checked through exact
    properties: a b = b a, (a1 + a2) b = a1 b + a2 b (mod q), and direct coefficient sums at
    one index each."""
    n, limbs, seed = point["N"], point["L"], point["seed"]
    q = inputs.random_modulus(limbs, seed)
    qi = inputs.to_int(q)
    instances = [inputs.instance(n, limbs, seed, index)[1:] for index in range(1, 4)]
    with fpc.Plan(n, 32 * limbs, limbs, q) as plan:
        products = [plan.run(a, b) for a, b in instances]
        (a1, b1), (a2, _), _ = instances
        assert np.array_equal(plan.run(b1, a1), products[0])
        a12 = inputs.poly_from_ints([(x + y) % qi for x, y in zip(inputs.poly_to_ints(a1), inputs.poly_to_ints(a2))],
                                    limbs)
        sum_product = inputs.poly_to_ints(plan.run(a12, b1))
        a2b1 = inputs.poly_to_ints(plan.run(a2, b1))
    c1 = inputs.poly_to_ints(products[0])
    assert sum_product == [(x + y) % qi for x, y in zip(c1, a2b1)]
    for (a, b), c, i in zip(instances, products, (1, n // 3, n - 2)):
        assert np.array_equal(oracle.schoolbook_at(q, a, b, i)[0], c[i]), i


@pytest.mark.parametrize("points", big_configs(), ids=lambda ps: f"N{ps[0]['N']}_L{ps[0]['L']}")
def test_full_size_against_reference_hashes(points, fpc, inputs):
    """Every hashed instance and edge pair of N=32768/L=868 and N=65536/L=1747, bit-exact
    against the reference checker's SHA-256 (tests/golden/baseline_cfg.json)."""
    checked = 0
    for point in points:
        n, limbs = point["N"], point["L"]
        plan = None
        try:
            for label, q, a, b, entry in baseline_cases(point, inputs):
                assert cases.sha256(a.astype("<u4").tobytes()) == entry["a_sha256"], label
                assert cases.sha256(b.astype("<u4").tobytes()) == entry["b_sha256"], label
                if plan is None:
                    plan = fpc.Plan(n, 32 * limbs, limbs, q)
                    assert plan.info()["gemm"] == 3  # both byte GEMMs on tensor cores
                c = plan.run(a, b)
                assert cases.sha256(c.tobytes()) == entry["c_sha256"], (point["seed"], label)
                checked += 1
        finally:
            if plan is not None:
                plan.close()
    assert checked == sum(len(p["cases"]) for p in points)


@pytest.mark.parametrize("point", first_points(), ids=lambda p: f"N{p['N']}_L{p['L']}")
def test_full_size_properties(point, fpc, inputs, oracle):
    """Size-independent checks on the first hashed instance: direct coefficient sums at both
    ends, and the negacyclic shift a*(X b) = X (a b)."""
    n, limbs = point["N"], point["L"]
    label, q, a, b, entry = next(iter(baseline_cases(point, inputs)))
    with fpc.Plan(n, 32 * limbs, limbs, q) as plan:
        c = plan.run(a, b)
        assert cases.sha256(c.tobytes()) == entry["c_sha256"], label
        for i in (0, n - 1):
            assert np.array_equal(oracle.schoolbook_at(q, a, b, i)[0], c[i]), i
        # negacyclic shift: X*b has b_{N-1} negated at index 0
        qi = inputs.to_int(q)
        xb = np.roll(b, 1, axis=0)
        xb[0] = inputs.from_int((qi - inputs.to_int(b[-1])) % qi, limbs)
        shifted = plan.run(a, xb)
    assert np.array_equal(shifted[1:], c[:-1])
    assert inputs.to_int(shifted[0]) == (qi - inputs.to_int(c[-1])) % qi
