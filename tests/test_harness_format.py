"""The platform's on-disk point format, and the drop-in at the binary level.

CPU: a point directory written here has exactly the files and manifest keys the
platform harness reads (src/main.cpp:137-151: "N", "W", "L", "cases" scanned
from manifest.json; point/q.bin of L words; cases/NNNNNN/{a,b}.bin of N*L words).
GPU: the reference's own, unmodified harness src/main.cpp, linked against this
library's fherma_init/run/free (built by oracle/build_ref.sh into
oracle/_ref/harness_b200), answers a point directory bit-exactly.
"""
import importlib.util
import json
import os
import subprocess

import numpy as np
import pytest

import cases
from conftest import PACKAGE_DIR, REPO
from test_oracle import point_pairs, reference_points


@pytest.fixture(scope="module")
def harness():
    spec = importlib.util.spec_from_file_location("fpc_b200_harness", os.path.join(PACKAGE_DIR, "harness.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def reference_point_dir(harness, tmp_path, inputs, index=7):
    point = reference_points()[index]  # N=1024, W=512 bits (16 limbs)
    q, pairs = point_pairs(point)
    limbs = point["L"]
    arrays = [(np.frombuffer(cases.pack(a, limbs), "<u4").reshape(-1, limbs),
               np.frombuffer(cases.pack(b, limbs), "<u4").reshape(-1, limbs)) for a, b in pairs]
    root = harness.write_point(tmp_path / "point", point["N"], point["W"], limbs, inputs.from_int(q, limbs), arrays)
    return root, point


def test_point_directory_layout(harness, tmp_path, inputs):
    root, point = reference_point_dir(harness, tmp_path, inputs)
    manifest = json.loads((root / "manifest.json").read_text())
    assert manifest == {"point": {"N": point["N"], "W": point["W"], "L": point["L"]}, "cases": len(point["cases"])}
    assert (root / "point" / "q.bin").stat().st_size == 4 * point["L"]
    for i, expect in enumerate(point["cases"]):
        a = (root / "cases" / f"{i:06d}" / "a.bin").read_bytes()
        assert cases.sha256(a) == expect["a_sha256"]
    p, q, count, case = harness.read_point(root)
    assert count == len(point["cases"]) and case(0)[0].shape == (point["N"], point["L"])


@pytest.mark.gpu
def test_python_runner_answers_a_point(harness, tmp_path, inputs):
    root, point = reference_point_dir(harness, tmp_path, inputs)
    results = harness.run_point(root)
    assert [c["status"] for c in results["cases"]] == ["ok"] * len(point["cases"])
    assert harness.output_hashes(root) == [c["c_sha256"] for c in point["cases"]]


@pytest.mark.gpu
def test_reference_harness_links_and_answers(harness, tmp_path, inputs):
    binary = os.path.join(REPO, "oracle", "_ref", "harness_b200")
    if not os.path.exists(binary):
        pytest.skip("oracle/_ref not built (needs the reference sources at build time)")
    root, point = reference_point_dir(harness, tmp_path, inputs)
    subprocess.run([binary, str(root)], check=True, timeout=300)
    results = harness.read_results(root)
    assert [c["status"] for c in results["cases"]] == ["ok"] * len(point["cases"])
    assert harness.output_hashes(root) == [c["c_sha256"] for c in point["cases"]]


@pytest.mark.gpu
@pytest.mark.parametrize("index", [7, 10])  # N=1024/W=512, and N=65536/W=1747 bits (the reference's main point)
def test_reference_binary_and_this_library_agree(harness, tmp_path, inputs, index):
    """The reference's original CUDA solution (src/solve.cu + src/main.cpp, built for sm_100a)
    and this library behind the same unmodified harness answer the reference checker's cases
    identically; both harnesses' per-case fherma_run times are printed for comparison."""
    solution = os.path.join(REPO, "oracle", "_ref", "solution")
    ours = os.path.join(REPO, "oracle", "_ref", "harness_b200")
    if not (os.path.exists(solution) and os.path.exists(ours)):
        pytest.skip("oracle/_ref not built (needs the reference sources at build time)")
    root, point = reference_point_dir(harness, tmp_path, inputs, index)
    timings = {}
    for name, binary in (("reference", solution), ("b200", ours)):
        out = root / "out"
        if out.exists():
            for f in sorted(out.rglob("*"), reverse=True):
                f.unlink() if f.is_file() else f.rmdir()
        subprocess.run([binary, str(root)], check=True, timeout=600)
        results = harness.read_results(root)
        assert [c["status"] for c in results["cases"]] == ["ok"] * len(point["cases"]), name
        assert harness.output_hashes(root) == [c["c_sha256"] for c in point["cases"]], name
        timings[name] = {"init_s": results["init_s"], "case_ms": [round(1000 * c["seconds"], 3) for c in results["cases"]]}
    print(json.dumps({"point": {"N": point["N"], "W": point["W"]}, **timings}))
