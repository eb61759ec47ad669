"""Regenerates the reference checker's operand pairs (test infrastructure).

The reference writes its cases with Python's `random` module and a fixed set of
edge pairs; these functions restate that generation so the committed golden
fixtures (hashes of the reference's own outputs) can be checked without the
reference checkout:

  reference_pairs   tests/reference.py:50-60   (edge pairs, then one random pair per seed)
  stress_pairs      tools/stress_local.py:21-27 (wrap, alternating, limb boundary, halves)
  modulus           tests/reference.py:9-16    (largest prime q < 2^width with q = 1 mod 2N)
"""
from __future__ import annotations

import hashlib
import random


def is_probable_prime(n: int) -> bool:
    """Miller-Rabin with the first 40 primes as bases (stands in for gmpy2.is_prime(n, 40))."""
    if n < 2:
        return False
    small = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73,
             79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149, 151, 157, 163,
             167, 173]
    for p in small:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def modulus(n: int, width: int) -> int:
    step = 2 * n
    q = ((1 << width) - 2) // step * step + 1
    while q > 1 and not is_probable_prime(q):
        q -= step
    if q <= 1:
        raise ValueError("no modulus for this point")
    return q


def reference_pairs(n: int, q: int, seeds, edge_cases: bool = True):
    pairs = []
    if edge_cases:
        zeros, ones, maximum = [0] * n, [1] * n, [q - 1] * n
        impulse, shifted = zeros.copy(), zeros.copy()
        impulse[0] = 1
        shifted[-1] = q - 1
        pairs += [(zeros, maximum), (ones, maximum), (maximum, maximum), (impulse, shifted)]
    for seed in seeds:
        rng = random.Random(seed)
        a = [rng.randrange(q) for _ in range(n)]
        b = [rng.randrange(q) for _ in range(n)]
        pairs.append((a, b))
    return pairs


def stress_pairs(n: int, q: int, width: int):
    limbs = (width + 31) // 32
    last = [0] * n
    last[-1] = q - 1
    ones = [1] * n
    alternating = [q - 1 if i % 2 else 0 for i in range(n)]
    boundaries = [min(q - 1, (1 << (32 * (i % limbs + 1))) - 1) for i in range(n)]
    return [(last, last), (alternating, ones), (boundaries, boundaries), ([q // 2] * n, [q // 2 + 1] * n)]


def pack(values, limbs: int) -> bytes:
    return b"".join(int(v).to_bytes(4 * limbs, "little") for v in values)


def sha256(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()
