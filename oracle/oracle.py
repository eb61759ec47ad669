"""CPU oracle loader — TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg may import this
module, and only as the checker / baseline, never as the thing measured.

  kronecker(q, a, b)        GMP Kronecker product (liboracle.so, restates
                            the reference's tests/reference.py:29-43)
  schoolbook_at(q, a, b, i) exact coefficients i..i+count-1 by direct GMP sums
                            (tests/reference.py:19-26, one coefficient at a time)
  kronecker_python / schoolbook_python: the same two algorithms over Python
                            ints, for tiny cases (independent of GMP)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", HERE, "-s"], check=True)


def library() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            build()
        lib = ctypes.CDLL(LIBRARY)
        u32, p = ctypes.c_uint32, ctypes.c_void_p
        lib.oracle_negacyclic_kronecker.argtypes = [u32, u32, p, p, p, p]
        lib.oracle_negacyclic_schoolbook.argtypes = [u32, u32, p, p, p, p, u32, u32]
        lib.oracle_slot_bytes.argtypes = [u32, u32, p]
        lib.oracle_slot_bytes.restype = ctypes.c_size_t
        _lib = lib
    return _lib


def _prep(q, a, b):
    q = np.ascontiguousarray(q, dtype=np.uint32)
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    assert a.shape == b.shape and a.shape[1] == q.shape[0]
    return q, a, b


def kronecker(q, a, b) -> np.ndarray:
    q, a, b = _prep(q, a, b)
    n, limbs = a.shape
    c = np.zeros_like(a)
    status = library().oracle_negacyclic_kronecker(n, limbs, q.ctypes.data, a.ctypes.data, b.ctypes.data,
                                                   c.ctypes.data)
    if status != 0:
        raise ValueError("oracle: q must be nonzero")
    return c


def schoolbook_at(q, a, b, first: int, count: int = 1) -> np.ndarray:
    """Rows first..first+count-1 of the product, by direct sums (O(N) big products each)."""
    q, a, b = _prep(q, a, b)
    n, limbs = a.shape
    c = np.zeros_like(a)
    library().oracle_negacyclic_schoolbook(n, limbs, q.ctypes.data, a.ctypes.data, b.ctypes.data, c.ctypes.data,
                                           first, count)
    return c[first:first + count]


def kronecker_python(a: list, b: list, q: int) -> list:
    n = len(a)
    stride = ((n * (q - 1) ** 2).bit_length() + 7) // 8 or 1
    left = int.from_bytes(b"".join(x.to_bytes(stride, "little") for x in a), "little")
    right = int.from_bytes(b"".join(x.to_bytes(stride, "little") for x in b), "little")
    raw = (left * right).to_bytes(2 * n * stride, "little")
    return [(int.from_bytes(raw[i * stride:(i + 1) * stride], "little")
             - int.from_bytes(raw[(i + n) * stride:(i + n + 1) * stride], "little")) % q for i in range(n)]


def schoolbook_python(a: list, b: list, q: int) -> list:
    n = len(a)
    out = [0] * n
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            if i + j < n:
                out[i + j] += x * y
            else:
                out[i + j - n] -= x * y
    return [v % q for v in out]
