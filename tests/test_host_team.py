"""The host path's copy team on CPU (no GPU): builds tests/native/host_team_check.cpp against
fherma-polynomial-cuda_b200/csrc/host_io.h and runs it with several team sizes. It packs
transform-ordered chunks with per-chunk counters consumed in order by a launcher thread,
unpacks chunks as they are marked landed, and repeats 300 calls with idle gaps, so a lost
wake-up or a chunk released before all workers finished shows up as a failure or a timeout."""
import os
import subprocess

import pytest

from conftest import REPO


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    out = tmp_path_factory.mktemp("host_team") / "host_team_check"
    source = os.path.join(REPO, "tests", "native", "host_team_check.cpp")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", source, "-o", str(out)], check=True)
    return str(out)


@pytest.mark.parametrize("workers", [1, 3, 12])
def test_host_team_packs_and_unpacks_in_order(checker, workers):
    done = subprocess.run([checker, str(workers)], capture_output=True, text=True, timeout=120)
    assert done.returncode == 0, done.stderr + done.stdout
    assert "0 failures" in done.stdout
