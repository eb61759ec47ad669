"""Writes tests/golden/*.json from the reference's own checker code.

Run with REFERENCE set to a checkout of the reference project (required):

    REFERENCE=<checkout> python tests/golden/make_golden.py [--big --jobs J]

It imports the reference's tests/reference.py and calls its `save_point`,
`kronecker` and `modulus` functions. That module imports gmpy2, which this
image lacks; a stand-in module is installed under that name first: `mpz` is a
Python int whose multiplication calls GMP's mpz_mul through ctypes (the same
library gmpy2 wraps), and `is_prime` is Miller-Rabin over the first 40 prime
bases. Nothing else of the reference is changed or copied.

Outputs (hashes of the reference's bytes; full values only for tiny points):
  reference_points.json  tools/validate_local.py:13-14 points, tools/stress_local.py:16 points
  baseline_cfg.json      the N=4096/L=64 random-odd-q product and its edge pairs; --big adds
                         N=32768/L=868 (q from seed 1, operand indices 0..19, every edge pair)
                         and N=65536/L=1747 (seeds 2..21, one instance each; every edge pair
                         with the seed-2 q). The big products run in parallel worker processes
                         (--jobs; about 10 GB of memory each at N=65536/L=1747) and are cached
                         in --cache as they finish, so an interrupted run resumes.
"""
from __future__ import annotations

import argparse
import ctypes
import multiprocessing
import importlib.util
import json
import os
import sys
import tempfile
import time
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(HERE))
import cases  # noqa: E402

REFERENCE = Path(os.environ["REFERENCE"]) if os.environ.get("REFERENCE") else None

_gmp = ctypes.CDLL("libgmp.so.10")


class _MpzStruct(ctypes.Structure):
    _fields_ = [("alloc", ctypes.c_int), ("size", ctypes.c_int), ("d", ctypes.c_void_p)]


def _gmp_mul(x: int, y: int) -> int:
    if x == 0 or y == 0:
        return 0
    za, zb, zc = _MpzStruct(), _MpzStruct(), _MpzStruct()
    for z in (za, zb, zc):
        _gmp.__gmpz_init(ctypes.byref(z))
    try:
        for z, v in ((za, x), (zb, y)):
            raw = v.to_bytes((v.bit_length() + 7) // 8, "little")
            _gmp.__gmpz_import(ctypes.byref(z), ctypes.c_size_t(len(raw)), -1, ctypes.c_size_t(1), 0,
                               ctypes.c_size_t(0), raw)
        _gmp.__gmpz_mul(ctypes.byref(zc), ctypes.byref(za), ctypes.byref(zb))
        bits = (x.bit_length() + y.bit_length() + 7) // 8 + 8
        out = ctypes.create_string_buffer(bits)
        count = ctypes.c_size_t(0)
        _gmp.__gmpz_export(out, ctypes.byref(count), -1, ctypes.c_size_t(1), 0, ctypes.c_size_t(0),
                           ctypes.byref(zc))
        return int.from_bytes(out.raw[:count.value], "little")
    finally:
        for z in (za, zb, zc):
            _gmp.__gmpz_clear(ctypes.byref(z))


class _Mpz(int):
    """int whose products go through GMP, like gmpy2.mpz."""

    def __mul__(self, other):
        return _Mpz(_gmp_mul(int(self), int(other)))

    __rmul__ = __mul__


def load_reference():
    if REFERENCE is None or not (REFERENCE / "tests/reference.py").exists():
        raise SystemExit("set REFERENCE to a checkout of the reference project (it must hold tests/reference.py)")
    stand_in = types.ModuleType("gmpy2")
    stand_in.mpz = _Mpz
    stand_in.is_prime = lambda n, reps=25: cases.is_probable_prime(int(n))
    sys.modules["gmpy2"] = stand_in
    spec = importlib.util.spec_from_file_location("fherma_reference_checker", REFERENCE / "tests/reference.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def record(n, width, limbs, q, pairs, outputs, full_limit=4096):
    out = []
    for (a, b), c in zip(pairs, outputs):
        entry = {"a_sha256": cases.sha256(cases.pack(a, limbs)),
                 "b_sha256": cases.sha256(cases.pack(b, limbs)),
                 "c_sha256": cases.sha256(c)}
        if n * limbs <= full_limit:
            entry["c_hex"] = c.hex()
        out.append(entry)
    return out


def validate_points(ref):
    points = []
    # tools/validate_local.py:13-14, seeds (101, 202) and edge cases
    for n, width in [(1, 2), (2, 5), (8, 16), (64, 31), (64, 33), (128, 128), (256, 256),
                     (1024, 512), (8192, 256), (32768, 868), (65536, 1747)]:
        started = time.time()
        with tempfile.TemporaryDirectory() as tmp:
            info = ref.save_point(tmp, n, width, seeds=(101, 202), edge_cases=True)
            limbs = info["L"]
            q = int.from_bytes((Path(tmp) / "point/q.bin").read_bytes(), "little")
            outputs = [(Path(tmp) / "reference" / f"{i:06d}" / "c.bin").read_bytes() for i in range(info["cases"])]
            pairs = cases.reference_pairs(n, q, (101, 202), True)
            for i, (a, b) in enumerate(pairs):  # the regeneration must match the reference's files
                assert (Path(tmp) / "cases" / f"{i:06d}" / "a.bin").read_bytes() == cases.pack(a, limbs)
                assert (Path(tmp) / "cases" / f"{i:06d}" / "b.bin").read_bytes() == cases.pack(b, limbs)
        points.append({"N": n, "W": width, "L": limbs, "q_hex": hex(q), "kind": "reference_pairs",
                       "seeds": [101, 202], "edge_cases": True,
                       "cases": record(n, width, limbs, q, pairs, outputs)})
        print(json.dumps({"N": n, "W": width, "cases": len(outputs), "s": round(time.time() - started, 1)}), flush=True)
    # tools/stress_local.py:16-27 (4 seeds at the two small stress points, 20 at the ranked points)
    for n, width, count in [(128, 4096, 4), (131072, 128, 4), (32768, 868, 20), (65536, 1747, 20)]:
        started = time.time()
        q = int(ref.modulus(n, width))
        limbs = (width + 31) // 32
        seeds = list(range(10001, 10001 + count))
        pairs = cases.reference_pairs(n, q, seeds, False) + cases.stress_pairs(n, q, width)
        outputs = [b"".join(int(x).to_bytes(4 * limbs, "little") for x in ref.kronecker(a, b, q)) for a, b in pairs]
        points.append({"N": n, "W": width, "L": limbs, "q_hex": hex(q), "kind": "stress_pairs",
                       "seeds": seeds, "edge_cases": False,
                       "cases": record(n, width, limbs, q, pairs, outputs)})
        print(json.dumps({"N": n, "W": width, "cases": len(outputs), "s": round(time.time() - started, 1)}), flush=True)
    return points


def _instance_task(task):
    """One big product through the reference's kronecker, in a worker process."""
    n, limbs, seed, label = task
    sys.path.insert(0, str(REPO / "fherma-polynomial-cuda_b200"))
    import inputs  # the package's seeded generator (numpy)
    ref = load_reference()
    started = time.time()
    if label.startswith("seed"):
        q, a, b = inputs.instance(n, limbs, seed, int(label.split("index")[1]))
    else:
        q = inputs.random_modulus(limbs, seed)
        x, y = _edge_names(inputs, label)
        a, b = inputs.edge_operand(n, q, x), inputs.edge_operand(n, q, y)
    entry = {"label": label,
             "a_sha256": cases.sha256(a.astype("<u4").tobytes()),
             "b_sha256": cases.sha256(b.astype("<u4").tobytes())}
    qi = inputs.to_int(q)
    a, b = inputs.poly_to_ints(a), inputs.poly_to_ints(b)
    c = ref.kronecker(a, b, qi)
    del a, b
    entry["c_sha256"] = cases.sha256(cases.pack(c, limbs))
    return {"N": n, "L": limbs, "seed": seed, "q_hex": hex(qi), "entry": entry, "s": round(time.time() - started, 1)}


def _edge_names(inputs, label):
    for x, y in inputs.EDGE_PAIRS:
        if label == f"edge_{x}_{y}":
            return x, y
    raise KeyError(label)


def _point_tasks(n, limbs, seed, instances, edges):
    sys.path.insert(0, str(REPO / "fherma-polynomial-cuda_b200"))
    import inputs
    tasks = [(n, limbs, s, f"seed{s}_index{i}") for s, i in instances]
    if edges:
        tasks += [(n, limbs, seed, f"edge_{x}_{y}") for x, y in inputs.EDGE_PAIRS]
    return tasks


def baseline_points(big, jobs, cache_path):
    # (N, L, seed of the edge pairs' q, [(seed, operand index)], edges)
    configs = [(4096, 64, 0, [(0, 0)], True)]
    if big:
        configs += [(32768, 868, 1, [(1, i) for i in range(20)], True),
                    (65536, 1747, 2, [(s, 0) for s in range(2, 22)], True)]
    tasks = [t for n, limbs, seed, inst, edges in configs for t in _point_tasks(n, limbs, seed, inst, edges)]
    done = {}
    cache = Path(cache_path)
    if cache.exists():
        for line in cache.read_text().splitlines():
            item = json.loads(line)
            done[(item["N"], item["L"], item["seed"], item["entry"]["label"])] = item
    todo = sorted((t for t in tasks if t not in done), key=lambda t: -t[0] * t[1])
    if todo:
        context = multiprocessing.get_context("spawn")
        with context.Pool(jobs, maxtasksperchild=1) as pool, cache.open("a") as log:
            for item in pool.imap_unordered(_instance_task, todo):
                done[(item["N"], item["L"], item["seed"], item["entry"]["label"])] = item
                log.write(json.dumps(item) + "\n")
                log.flush()
                print(json.dumps({"N": item["N"], "L": item["L"], "seed": item["seed"],
                                  "label": item["entry"]["label"], "s": item["s"]}), flush=True)
    points = {}
    for task in tasks:  # one point per (N, L, q seed), cases in task order
        item = done[task]
        key = (item["N"], item["L"], item["seed"])
        if key not in points:
            points[key] = {"N": item["N"], "L": item["L"], "seed": item["seed"], "q_hex": item["q_hex"], "cases": []}
        points[key]["cases"].append(item["entry"])
    return list(points.values())


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--big", action="store_true", help="add the N=32768/L=868 and N=65536/L=1747 products")
    parser.add_argument("--only", choices=("reference", "baseline"), default=None)
    parser.add_argument("--jobs", type=int, default=4, help="worker processes for the baseline products")
    parser.add_argument("--cache", default=os.path.join(tempfile.gettempdir(), "fherma_golden_cache.jsonl"),
                        help="finished baseline products, one JSON line each (resumes an interrupted run)")
    args = parser.parse_args()
    ref = load_reference()
    header = {"generated_by": "tests/golden/make_golden.py",
              "checker": "reference tests/reference.py (save_point, kronecker, modulus) with a GMP-backed gmpy2 stand-in"}
    if args.only in (None, "reference"):
        (HERE / "reference_points.json").write_text(json.dumps({**header, "points": validate_points(ref)}, indent=1) + "\n")
    if args.only in (None, "baseline"):
        (HERE / "baseline_cfg.json").write_text(json.dumps({**header, "points": baseline_points(args.big, args.jobs, args.cache)}, indent=1) + "\n")


if __name__ == "__main__":
    main()
