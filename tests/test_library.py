"""The C-ABI libraries load and export what the headers declare (no GPU calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PACKAGE_DIR, REPO


def declared(header):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(negacyclic_\w+)\s*\(", text)))


def exported(library):
    out = subprocess.run(["nm", "-D", "--defined-only", library], check=True, capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_c_abi_exports_every_declared_symbol(fpc):
    symbols = exported(fpc.LIBRARY)
    names = declared("negacyclic.h")
    assert names, "no declarations parsed"
    missing = [name for name in names if name not in symbols]
    assert not missing, missing
    assert set(names) == set(fpc.EXPORTED)
    lib = fpc.library()
    for name in names:
        assert getattr(lib, name) is not None


def test_fherma_shim_exports_plugin_entry_points():
    library = os.path.join(PACKAGE_DIR, "libfherma_negacyclic.so")
    demangled = subprocess.run(["nm", "-DC", "--defined-only", library], check=True, capture_output=True,
                               text=True).stdout
    for entry in ("fherma_init(fherma::Point const&)", "fherma_run(void*, fherma::Inputs const&)",
                  "fherma_free(void*)"):
        assert entry in demangled, entry
    ctypes.CDLL(library)  # resolves libnegacyclic.so through its rpath


def test_init_without_a_b200_fails_cleanly(fpc):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(RuntimeError, match="negacyclic_init"):
        fpc.Plan(16, 32, 1, np.array([97], np.uint32))


def test_invalid_point_is_rejected_before_touching_the_device(fpc):
    with pytest.raises(RuntimeError, match=r"L must equal \(W \+ 31\) / 32"):
        fpc.Plan(16, 64, 1, np.array([97], np.uint32))
    with pytest.raises(RuntimeError, match="q must hold L words"):
        fpc.Plan(16, 32, 1, np.array([97, 1], np.uint32))


def test_product_path_has_no_cpu_fallback():
    """The package never imports the oracle: the product path is the CUDA library or an error."""
    for name in os.listdir(PACKAGE_DIR):
        if name.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
            text = open(os.path.join(PACKAGE_DIR, name)).read()
            assert "oracle" not in text.lower(), name
    csrc = os.path.join(PACKAGE_DIR, "csrc")
    for name in os.listdir(csrc):
        text = open(os.path.join(csrc, name)).read()
        assert "oracle" not in text.lower() and "gmp" not in text.lower(), name
