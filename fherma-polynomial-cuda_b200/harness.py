"""On-disk point directories of the FHERMA runner, and a runner over this library.

Format (the platform harness, src/main.cpp:1-15, 137-209; tests/reference.py:63-75):

    manifest.json            {"point": {"N": n, "W": w, "L": limbs}, "cases": k}
    point/q.bin              q, limbs little-endian uint32 words
    cases/NNNNNN/a.bin       [N][L] uint32 little-endian
    cases/NNNNNN/b.bin
    out/NNNNNN/c.bin         written by the solution
    out/results.json         {"init_s": t, "cases": [{"i", "seconds", "status"[, "note"]}]}

    python harness.py make DIR --n N --limbs L [--seed S] [--cases K]   random odd q, seeded cases
    python harness.py run DIR                                            this library (C ABI)
    python harness.py hashes DIR                                         SHA-256 of every out/*/c.bin
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _inputs():
    spec = importlib.util.spec_from_file_location("fpc_b200_inputs", os.path.join(HERE, "inputs.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def write_point(directory, n: int, w: int, limbs: int, q, pairs) -> Path:
    """Writes a point directory: q ([L] uint32) and operand pairs ([N][L] uint32 each)."""
    root = Path(directory)
    (root / "point").mkdir(parents=True, exist_ok=True)
    np.ascontiguousarray(q, dtype="<u4").tofile(root / "point" / "q.bin")
    for i, (a, b) in enumerate(pairs):
        case = root / "cases" / f"{i:06d}"
        case.mkdir(parents=True, exist_ok=True)
        for name, x in (("a", a), ("b", b)):
            x = np.ascontiguousarray(x, dtype="<u4")
            assert x.shape == (n, limbs)
            x.tofile(case / f"{name}.bin")
    (root / "manifest.json").write_text(json.dumps({"point": {"N": n, "W": w, "L": limbs}, "cases": len(pairs)}))
    return root


def read_point(directory):
    root = Path(directory)
    manifest = json.loads((root / "manifest.json").read_text())
    point = manifest["point"]
    n, limbs = int(point["N"]), int(point["L"])
    q = np.fromfile(root / "point" / "q.bin", dtype="<u4")
    if q.shape != (limbs,):
        raise ValueError("q: wrong size")

    def case(i):
        d = root / "cases" / f"{i:06d}"
        a = np.fromfile(d / "a.bin", dtype="<u4")
        b = np.fromfile(d / "b.bin", dtype="<u4")
        if a.size != n * limbs or b.size != n * limbs:
            raise ValueError(f"case {i}: wrong size")
        return a.reshape(n, limbs), b.reshape(n, limbs)

    return point, q, int(manifest["cases"]), case


def read_results(directory) -> dict:
    return json.loads((Path(directory) / "out" / "results.json").read_text())


def output(directory, i: int, n: int, limbs: int) -> np.ndarray:
    return np.fromfile(Path(directory) / "out" / f"{i:06d}" / "c.bin", dtype="<u4").reshape(n, limbs)


def output_hashes(directory) -> list[str]:
    out = Path(directory) / "out"
    return [hashlib.sha256((d / "c.bin").read_bytes()).hexdigest()
            for d in sorted(out.iterdir()) if d.is_dir()]


def run_point(directory) -> dict:
    """What the platform harness does, through this library's C ABI: init once (timed),
    then every case (fherma_run timed alone), writing out/ and out/results.json."""
    spec = importlib.util.spec_from_file_location("fpc_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    fpc = sys.modules.get("fpc_b200")
    if fpc is None:
        fpc = importlib.util.module_from_spec(spec)
        sys.modules["fpc_b200"] = fpc
        spec.loader.exec_module(fpc)
    point, q, count, case = read_point(directory)
    out = Path(directory) / "out"
    out.mkdir(exist_ok=True)
    started = time.perf_counter()
    state = fpc.fherma_init(fpc.Point(int(point["N"]), int(point["W"]), int(point["L"]), q))
    init_s = time.perf_counter() - started
    cases = []

    def report():
        (out / "results.json").write_text(json.dumps({"init_s": init_s, "cases": cases}))

    report()
    try:
        for i in range(count):
            try:
                a, b = case(i)
                t0 = time.perf_counter()
                c = fpc.fherma_run(state, fpc.Inputs(a, b)).c
                seconds = time.perf_counter() - t0
                (out / f"{i:06d}").mkdir(exist_ok=True)
                c.astype("<u4").tofile(out / f"{i:06d}" / "c.bin")
                cases.append({"i": i, "seconds": seconds, "status": "ok"})
            except Exception as failure:  # recorded per case, as the platform harness does
                cases.append({"i": i, "seconds": None, "status": "crashed", "note": str(failure)[:200]})
            report()
    finally:
        fpc.fherma_free(state)
    return {"init_s": init_s, "cases": cases}


def make_point(directory, n: int, limbs: int, seed: int, cases: int):
    inputs = _inputs()
    q = inputs.random_modulus(limbs, seed)
    pairs = [inputs.instance(n, limbs, seed, i)[1:] for i in range(cases)]
    return write_point(directory, n, 32 * limbs, limbs, q, pairs)


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    parser.add_argument("mode", choices=("make", "run", "hashes"))
    parser.add_argument("directory")
    parser.add_argument("--n", type=int, default=4096)
    parser.add_argument("--limbs", type=int, default=64)
    parser.add_argument("--seed", type=int, default=0)
    parser.add_argument("--cases", type=int, default=2)
    args = parser.parse_args()
    if args.mode == "make":
        make_point(args.directory, args.n, args.limbs, args.seed, args.cases)
    elif args.mode == "run":
        print(json.dumps(run_point(args.directory)))
    else:
        print("\n".join(output_hashes(args.directory)))


if __name__ == "__main__":
    main()
