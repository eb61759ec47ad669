"""The streamed host path's chunk lists on CPU (no GPU): builds tests/native/host_chunks_check.cpp
against fherma-polynomial-cuda_b200/csrc/host_chunks.h and runs it over every N = 2^0..2^17,
every ring split with N/s <= 8192 and limb counts on both sides of the wide-row threshold. It
checks the per-direction chunk budget, that the input chunks cover every coefficient of both
operands exactly once (operand a before b for narrow rows), and that the output chunks tile [0, N)
on the boundaries their transposes need."""
import os
import subprocess

from conftest import REPO


def test_chunk_lists_cover_every_coefficient_within_budget(tmp_path):
    binary = tmp_path / "host_chunks_check"
    source = os.path.join(REPO, "tests", "native", "host_chunks_check.cpp")
    subprocess.run(["g++", "-O2", "-std=c++17", source, "-o", str(binary)], check=True)
    done = subprocess.run([str(binary)], capture_output=True, text=True, timeout=120)
    assert done.returncode == 0, done.stderr + done.stdout
    assert "0 failures" in done.stdout
