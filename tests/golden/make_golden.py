"""Writes tests/golden/*.json from the reference's own checker code.

Run in a checkout that has the reference at REFERENCE (default /root/reference):

    python tests/golden/make_golden.py [--big]

It imports the reference's tests/reference.py and calls its `save_point`,
`kronecker` and `modulus` functions. That module imports gmpy2, which this
image lacks; a stand-in module is installed under that name first: `mpz` is a
Python int whose multiplication calls GMP's mpz_mul through ctypes (the same
library gmpy2 wraps), and `is_prime` is Miller-Rabin over the first 40 prime
bases. Nothing else of the reference is changed or copied.

Outputs (hashes of the reference's bytes; full values only for tiny points):
  reference_points.json  tools/validate_local.py:13-14 points, tools/stress_local.py:16 points
  baseline_cfg.json      the N=4096/L=64 random-odd-q product and its edge pairs
                         (--big adds one N=32768/L=868 and one N=65536/L=1747 instance)
"""
from __future__ import annotations

import argparse
import ctypes
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

REFERENCE = Path(os.environ.get("REFERENCE", "/root/reference"))

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
    # tools/stress_local.py:16-27 (4 seeds at the two small stress points, 2 at the ranked points)
    for n, width, count in [(128, 4096, 4), (131072, 128, 4), (32768, 868, 2), (65536, 1747, 2)]:
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


def baseline_points(ref, big):
    sys.path.insert(0, str(REPO / "fherma-polynomial-cuda_b200"))
    import inputs  # the package's seeded generator (numpy)
    configs = [(4096, 64, 0, [0], True)]
    if big:
        configs += [(32768, 868, 1, [0], False), (65536, 1747, 2, [0], False)]
    points = []
    for n, limbs, seed, indices, edges in configs:
        started = time.time()
        entries = []
        for index in indices:
            q, a, b = inputs.instance(n, limbs, seed, index)
            qi = inputs.to_int(q)
            c = ref.kronecker(inputs.poly_to_ints(a), inputs.poly_to_ints(b), qi)
            entries.append({"label": f"seed{seed}_index{index}",
                            "a_sha256": cases.sha256(a.astype("<u4").tobytes()),
                            "b_sha256": cases.sha256(b.astype("<u4").tobytes()),
                            "c_sha256": cases.sha256(cases.pack(c, limbs))})
        if edges:
            q = inputs.random_modulus(limbs, seed)
            qi = inputs.to_int(q)
            ops = inputs.edge_operands(n, q)
            for x, y in inputs.EDGE_PAIRS:
                c = ref.kronecker(inputs.poly_to_ints(ops[x]), inputs.poly_to_ints(ops[y]), qi)
                entries.append({"label": f"edge_{x}_{y}",
                                "a_sha256": cases.sha256(ops[x].astype("<u4").tobytes()),
                                "b_sha256": cases.sha256(ops[y].astype("<u4").tobytes()),
                                "c_sha256": cases.sha256(cases.pack(c, limbs))})
        points.append({"N": n, "L": limbs, "seed": seed, "q_hex": hex(inputs.to_int(inputs.random_modulus(limbs, seed))),
                       "cases": entries})
        print(json.dumps({"N": n, "L": limbs, "cases": len(entries), "s": round(time.time() - started, 1)}), flush=True)
    return points


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--big", action="store_true", help="add the N=32768/L=868 and N=65536/L=1747 products")
    parser.add_argument("--only", choices=("reference", "baseline"), default=None)
    args = parser.parse_args()
    ref = load_reference()
    header = {"generated_by": "tests/golden/make_golden.py",
              "checker": "reference tests/reference.py (save_point, kronecker, modulus) with a GMP-backed gmpy2 stand-in"}
    if args.only in (None, "reference"):
        (HERE / "reference_points.json").write_text(json.dumps({**header, "points": validate_points(ref)}, indent=1) + "\n")
    if args.only in (None, "baseline"):
        (HERE / "baseline_cfg.json").write_text(json.dumps({**header, "points": baseline_points(ref, args.big)}, indent=1) + "\n")


if __name__ == "__main__":
    main()
