"""The CPU oracle, pinned against the reference checker's own outputs (no GPU).

tests/golden/*.json hold SHA-256 hashes (and, for tiny points, full values) of
operands and products written by the reference's tests/reference.py
(save_point / kronecker) — see tests/golden/make_golden.py. Here the operands
are regenerated from their seeds, checked against the recorded operand hashes,
multiplied by the oracle, and the product compared with the recorded one.
"""
import json
import os

import numpy as np
import pytest

import cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def reference_points():
    with open(os.path.join(GOLDEN, "reference_points.json")) as f:
        return json.load(f)["points"]


def baseline_points():
    path = os.path.join(GOLDEN, "baseline_cfg.json")
    if not os.path.exists(path):  # written by make_golden.py; required in a full checkout
        return []
    with open(path) as f:
        return json.load(f)["points"]


def point_pairs(point):
    q = int(point["q_hex"], 16)
    n, width = point["N"], point["W"]
    if point["kind"] == "reference_pairs":
        pairs = cases.reference_pairs(n, q, point["seeds"], point["edge_cases"])
    else:
        pairs = cases.reference_pairs(n, q, point["seeds"], False) + cases.stress_pairs(n, q, width)
    return q, pairs


def as_array(values, limbs):
    return np.frombuffer(cases.pack(values, limbs), dtype="<u4").reshape(len(values), limbs)


def point_id(point):
    return f"N{point['N']}_W{point['W']}_{point['kind']}"


@pytest.mark.parametrize("point", reference_points(), ids=point_id)
def test_oracle_matches_reference_checker(point, oracle, inputs):
    q, pairs = point_pairs(point)
    limbs = point["L"]
    assert len(pairs) == len(point["cases"])
    q_arr = inputs.from_int(q, limbs)
    for (a, b), expect in zip(pairs, point["cases"]):
        a_arr, b_arr = as_array(a, limbs), as_array(b, limbs)
        assert cases.sha256(a_arr.tobytes()) == expect["a_sha256"]
        assert cases.sha256(b_arr.tobytes()) == expect["b_sha256"]
        c = oracle.kronecker(q_arr, a_arr, b_arr)
        if "c_hex" in expect:
            assert c.tobytes().hex() == expect["c_hex"]
        assert cases.sha256(c.tobytes()) == expect["c_sha256"]


@pytest.mark.parametrize("point", baseline_points(), ids=lambda p: f"N{p['N']}_L{p['L']}")
def test_oracle_matches_reference_on_baseline_configs(point, oracle, inputs):
    if point["N"] * point["L"] > 4096 * 64:
        pytest.skip("full-size products are checked on the GPU side against the same hashes")
    n, limbs, seed = point["N"], point["L"], point["seed"]
    q = inputs.random_modulus(limbs, seed)
    assert hex(inputs.to_int(q)) == point["q_hex"]
    edges = inputs.edge_operands(n, q)
    for entry in point["cases"]:
        label = entry["label"]
        if label.startswith("seed"):
            index = int(label.split("index")[1])
            _, a, b = inputs.instance(n, limbs, seed, index)
        else:
            x, y = edge_pair(inputs, label)
            a, b = edges[x], edges[y]
        assert cases.sha256(a.astype("<u4").tobytes()) == entry["a_sha256"], label
        assert cases.sha256(b.astype("<u4").tobytes()) == entry["b_sha256"], label
        c = oracle.kronecker(q, a, b)
        assert cases.sha256(c.tobytes()) == entry["c_sha256"], label


def edge_pair(inputs, label):
    """(x, y) of an 'edge_<x>_<y>' label (names may contain underscores)."""
    for x, y in inputs.EDGE_PAIRS:
        if label == f"edge_{x}_{y}":
            return x, y
    raise KeyError(label)


def test_oracle_agrees_with_python_restatements(oracle, inputs):
    rng = np.random.Generator(np.random.PCG64(7))
    for n, limbs in [(1, 1), (2, 3), (8, 2), (16, 5), (32, 1)]:
        q = inputs.random_modulus(limbs, int(rng.integers(1 << 30)))
        qi = inputs.to_int(q)
        a = inputs.random_operand(rng, n, q)
        b = inputs.random_operand(rng, n, q)
        la, lb = inputs.poly_to_ints(a), inputs.poly_to_ints(b)
        want = oracle.schoolbook_python(la, lb, qi)
        assert oracle.kronecker_python(la, lb, qi) == want
        assert inputs.poly_to_ints(oracle.kronecker(q, a, b)) == want
        assert inputs.poly_to_ints(oracle.schoolbook_at(q, a, b, 0, n)) == want


def test_schoolbook_spot_check_matches_kronecker(oracle, inputs):
    q, a, b = inputs.instance(256, 8, 3, 0)
    full = oracle.kronecker(q, a, b)
    for i in (0, 1, 127, 255):
        assert np.array_equal(oracle.schoolbook_at(q, a, b, i)[0], full[i])
