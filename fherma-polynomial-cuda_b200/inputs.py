"""Seeded synthetic operands for the negacyclic product.

Layout everywhere: a coefficient is `L` little-endian uint32 limbs, and a
polynomial is `[N][L]` uint32, coefficient-major (the layout of the
reference's `fherma::Tensor<uint32_t>` with shape {N, L}, src/fherma.h:34-41).

Generators (numpy PCG64, fully determined by the seed):
  random_modulus(L, seed)         q uniform in [2^(32L-32), 2^(32L)), odd, top limb != 0
  random_operand(rng, N, q)       coefficients uniform in [0, q) by rejection
  instance(N, L, seed, index)     (q, a, b): q from `seed`, operands from (seed, index)
Edge operands follow the reference's checker (tests/reference.py:52-57,
tools/stress_local.py:23-27) plus carry-boundary inputs.
"""
from __future__ import annotations

import numpy as np


def to_int(limbs) -> int:
    """Little-endian uint32 limbs -> Python int."""
    return int.from_bytes(np.ascontiguousarray(limbs, dtype="<u4").tobytes(), "little")


def from_int(value: int, limbs: int) -> np.ndarray:
    """Python int (0 <= value < 2^(32*limbs)) -> little-endian uint32 limbs."""
    return np.frombuffer(int(value).to_bytes(4 * limbs, "little"), dtype="<u4").copy()


def poly_from_ints(values, limbs: int) -> np.ndarray:
    """List of Python ints -> [N][L] uint32."""
    raw = b"".join(int(v).to_bytes(4 * limbs, "little") for v in values)
    return np.frombuffer(raw, dtype="<u4").reshape(len(values), limbs).copy()


def poly_to_ints(poly: np.ndarray) -> list[int]:
    poly = np.ascontiguousarray(poly, dtype="<u4")
    row = poly.shape[1] * 4
    raw = poly.tobytes()
    return [int.from_bytes(raw[i * row:(i + 1) * row], "little") for i in range(poly.shape[0])]


def random_modulus(limbs: int, seed: int) -> np.ndarray:
    """Uniform random odd q with a nonzero top limb (32*limbs bits wide)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    q = rng.integers(0, 1 << 32, size=limbs, dtype=np.uint64).astype(np.uint32)
    while q[-1] == 0:
        q[-1] = np.uint32(rng.integers(1, 1 << 32, dtype=np.uint64))
    q[0] |= np.uint32(1)
    return q


def _less_than(rows: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Row-wise big-integer comparison rows < q (both little-endian limbs)."""
    differs = rows != q[None, :]
    reversed_differs = differs[:, ::-1]
    any_diff = reversed_differs.any(axis=1)
    top = q.shape[0] - 1 - reversed_differs.argmax(axis=1)
    picked = rows[np.arange(rows.shape[0]), top]
    return any_diff & (picked < q[top])


def random_operand(rng: np.random.Generator, n: int, q: np.ndarray) -> np.ndarray:
    """[n][L] coefficients uniform in [0, q): top limb masked to q's top bit, then rejection."""
    limbs = q.shape[0]
    top = int(q[-1])
    mask = np.uint32((1 << top.bit_length()) - 1) if top else np.uint32(0)
    out = np.empty((n, limbs), dtype=np.uint32)
    todo = np.arange(n)
    while todo.size:
        rows = rng.integers(0, 1 << 32, size=(todo.size, limbs), dtype=np.uint64).astype(np.uint32)
        rows[:, -1] &= mask
        ok = _less_than(rows, q)
        out[todo[ok]] = rows[ok]
        todo = todo[~ok]
    return out


def instance(n: int, limbs: int, seed: int, index: int = 0):
    """(q, a, b) for one seeded product: q depends on `seed` only."""
    q = random_modulus(limbs, seed)
    rng = np.random.Generator(np.random.PCG64([seed, index + 1]))
    a = random_operand(rng, n, q)
    b = random_operand(rng, n, q)
    return q, a, b


EDGE_NAMES = ("zero", "ones", "max", "impulse0", "impulse_last", "alternating", "alt_zero", "carry",
              "boundary", "half", "half_up")


def edge_operand(n: int, q: np.ndarray, name: str) -> np.ndarray:
    """One edge input: zero, unit, all q-1, impulses, alternating q-1/q-2, carry boundaries."""
    limbs = q.shape[0]
    qi = to_int(q)
    zero = np.zeros((n, limbs), dtype=np.uint32)
    if name == "zero":
        return zero
    if name == "ones":
        zero[:, 0] = 1 if qi > 1 else 0
        return zero
    if name == "max":
        return np.tile(from_int(qi - 1, limbs), (n, 1))
    if name == "impulse0":
        zero[0] = from_int(1 % qi, limbs)
        return zero
    if name == "impulse_last":
        zero[-1] = from_int(qi - 1, limbs)
        return zero
    if name == "alternating":  # q-1 at even indices, q-2 at odd ones
        out = np.tile(from_int(qi - 1, limbs), (n, 1))
        out[1::2] = from_int(max(qi - 2, 0), limbs)
        return out
    if name == "alt_zero":  # q-1 at odd indices, 0 at even (tools/stress_local.py:25)
        zero[1::2] = from_int(qi - 1, limbs)
        return zero
    if name == "carry":
        # 0xFFFFFFFF limbs where the value stays below q: all-ones below q's top limb,
        # and q's top limb minus one on top (or all-ones on q-1's top when that is 0).
        ff = np.full(limbs, 0xFFFFFFFF, dtype=np.uint32)
        top = int(q[-1])
        if top > 1:
            ff[-1] = top - 1
            below = ff
        else:
            below = from_int(qi - 1, limbs)
        return np.tile(below, (n, 1))
    if name == "boundary":  # min(q-1, 2^(32*(i mod L + 1)) - 1) (tools/stress_local.py:26)
        rows = np.stack([from_int(min(qi - 1, (1 << (32 * (j + 1))) - 1), limbs) for j in range(min(limbs, n))])
        return rows[np.arange(n) % limbs] if n else zero
    if name == "half":
        return np.tile(from_int(qi // 2, limbs), (n, 1))
    if name == "half_up":
        return np.tile(from_int((qi // 2 + 1) % qi, limbs), (n, 1))
    raise KeyError(name)


def edge_operands(n: int, q: np.ndarray) -> dict[str, np.ndarray]:
    """Every edge input of `edge_operand`, by name."""
    return {name: edge_operand(n, q, name) for name in EDGE_NAMES}


EDGE_PAIRS = [
    ("zero", "max"), ("ones", "max"), ("max", "max"), ("impulse0", "impulse_last"),
    ("impulse_last", "impulse_last"), ("alt_zero", "ones"), ("alternating", "alternating"),
    ("carry", "carry"), ("boundary", "boundary"), ("half", "half_up"),
]
