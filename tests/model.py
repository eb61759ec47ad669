"""Exact integer model of the device pipeline (test infrastructure).

Mirrors, step for step, what the CUDA kernels compute, with Python integers,
so the algebra (constants, layouts, bounds) can be checked on the CPU against
a schoolbook product before any kernel runs, and so intermediate device
buffers can be compared stage by stage at small sizes.

Pipeline (s-way split of the ring, N' = N/s, r primes p = 1 mod 2N'):
  convert   G[row][4k+d] = sum_j byte_j(x_row) * byte_d(256^j mod p_k)   (u8 GEMM)
            res = REDC(sum_d G*256^d) = x * 2^-32 mod p
  forward   merged-psi Cooley-Tukey NTT per (op, k, t), natural -> bit-reversed
  pointwise C_v = sum_{t+u=v} mont(A_t,B_u) + zeta * sum_{t+u=v+s} mont(A_t,B_u)
  inverse   Gentleman-Sande per (k, v), then * F_k = R^3 N'^-1 (P/p_k)^-1
  crt       G[i][c] = sum_{k,d} byte_d(v_k) * byte_{c-d}(W_k),  W_k = M_k + 2^(32(L+2)) f_k
  reduce    V = sum_w dots_w 2^(32w);  T, D = V mod / div 2^(32(L+2));  K = (D + 2^63) >> 64
            T' = T + K*Rneg;  c = T' mod q by one Barrett quotient step + corrections
"""
from __future__ import annotations

from dataclasses import dataclass, field

R32 = 1 << 32
NTT_MAX = 8192
PRIME_LO, PRIME_HI = 1 << 30, 1 << 31


def is_prime32(n: int) -> bool:
    if n < 2:
        return False
    for p in (2, 3, 5, 7):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7):  # deterministic below 3,215,031,751
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


def bitrev(x: int, bits: int) -> int:
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


@dataclass
class Plan:
    n: int
    limbs: int
    q: int
    split: int
    n_sub: int
    primes: list = field(default_factory=list)
    psi: list = field(default_factory=list)


def choose_primes(n_sub: int, q: int, bound: int):
    step = 2 * n_sub
    p = (PRIME_HI - 2) // step * step + 1
    primes, product = [], 1
    while product <= bound:
        if p < PRIME_LO:
            return None
        if is_prime32(p) and q % p != 0:
            primes.append(p)
            product *= p
        p -= step
    return primes


def make_plan(n: int, limbs: int, q: int, split: int | None = None) -> Plan:
    assert n >= 1 and n & (n - 1) == 0 and q >= 2
    bound = 4 * n * (q - 1) ** 2
    s = split or max(1, n // NTT_MAX)
    while True:
        primes = choose_primes(n // s, q, bound)
        if primes is not None:
            break
        s *= 2
        assert s <= n
    plan = Plan(n, limbs, q, s, n // s, primes)
    for p in primes:
        g = 2
        while pow(g, (p - 1) // 2, p) != p - 1:
            g += 1
        psi = pow(g, (p - 1) // (2 * plan.n_sub), p)
        assert pow(psi, plan.n_sub, p) == p - 1
        plan.psi.append(psi)
    return plan


def redc(t: int, p: int) -> int:
    """Montgomery reduction t * 2^-32 mod p for t < p * 2^32 (additive form)."""
    assert 0 <= t < p * R32
    pinv = (-pow(p, -1, R32)) % R32
    m = (t % R32) * pinv % R32
    u = (t + m * p) >> 32
    return u - p if u >= p else u


def mont(a: int, b: int, p: int) -> int:
    return redc(a * b, p)


def shoup(a: int, w: int, p: int) -> int:
    """a*w mod p with w' = floor(w 2^32 / p); valid for a < 2^32, w < p < 2^31."""
    wq = (w << 32) // p
    quotient = (a * wq) >> 32
    r = (a * w - quotient * p) % R32
    assert r < 2 * p
    return r - p if r >= p else r


def twiddles(plan: Plan, k: int):
    p, psi, n = plan.primes[k], plan.psi[k], plan.n_sub
    bits = n.bit_length() - 1
    fwd = [pow(psi, bitrev(m, bits), p) for m in range(n)]
    inv = [pow(psi, -bitrev(m, bits), p) for m in range(n)]
    zeta = [pow(psi, 2 * bitrev(m, bits) + 1, p) for m in range(n)]
    return fwd, inv, zeta


def ntt_forward(a: list, fwd: list, p: int) -> list:
    a = list(a)
    n = len(a)
    t, m = n, 1
    while m < n:
        t //= 2
        for i in range(m):
            w = fwd[m + i]
            for j in range(2 * i * t, 2 * i * t + t):
                u, v = a[j], shoup(a[j + t], w, p)
                a[j], a[j + t] = (u + v) % p, (u - v) % p
        m *= 2
    return a


def ntt_inverse(a: list, inv: list, p: int) -> list:
    """Gentleman-Sande without the final 1/n (folded into F_k)."""
    a = list(a)
    n = len(a)
    t, m = 1, n
    while m > 1:
        h, j1 = m // 2, 0
        for i in range(h):
            w = inv[h + i]
            for j in range(j1, j1 + t):
                u, v = a[j], a[j + t]
                a[j], a[j + t] = (u + v) % p, shoup((u - v) % p, w, p)
            j1 += 2 * t
        t *= 2
        m = h
    return a


def crt_constants(plan: Plan):
    big_p = 1
    for p in plan.primes:
        big_p *= p
    q, L = plan.q, plan.limbs
    m_k = [(big_p // p) % q for p in plan.primes]
    f_k = [(1 << 64) // p for p in plan.primes]
    rneg = (-big_p) % q
    finish = [pow(R32, 3, p) * pow(plan.n_sub, -1, p) * pow((big_p // p) % p, -1, p) % p for p in plan.primes]
    shift_bits = 32 * (L + 2)
    weights = [m + (f << shift_bits) for m, f in zip(m_k, f_k)]
    return big_p, weights, rneg, finish


def byte(x: int, i: int) -> int:
    return (x >> (8 * i)) & 255 if i >= 0 else 0


def convert(plan: Plan, coeff: int, k: int) -> int:
    """Byte-sliced conversion of one coefficient for prime k, as the GEMM + epilogue do it."""
    p = plan.primes[k]
    nbytes = 4 * plan.limbs
    weights = [pow(256, j, p) for j in range(nbytes)]
    g = [sum(byte(coeff, j) * byte(weights[j], d) for j in range(nbytes)) for d in range(4)]
    assert all(x < (1 << 31) for x in g)
    s_sum = sum(x << (8 * d) for d, x in enumerate(g))
    return redc(s_sum, p)


def reduce_words(plan: Plan, dots: list, rneg: int) -> int:
    """Carry-save words -> canonical c (the reduce kernel's arithmetic)."""
    q, L = plan.q, plan.limbs
    value = sum(d << (32 * w) for w, d in enumerate(dots))
    shift_bits = 32 * (L + 2)
    t, d = value % (1 << shift_bits), value >> shift_bits
    k = (d + (1 << 63)) >> 64
    tp = t + k * rneg
    qb = q.bit_length()
    sh = qb - 64
    q_top = q >> sh if sh >= 0 else q << -sh
    t_top = tp >> sh if sh >= 0 else tp << -sh
    assert t_top < (1 << 112) and (1 << 63) <= q_top < (1 << 64)
    divisor = q_top + 1
    mu_low = ((1 << 128) // divisor) - (1 << 64)
    assert 0 <= mu_low < (1 << 64)
    th, tl = t_top >> 64, t_top & ((1 << 64) - 1)
    prod_l = tl * mu_low
    prod_h = th * mu_low
    word1 = (prod_l >> 64) + (prod_h & ((1 << 64) - 1))
    word2 = (prod_h >> 64) + (word1 >> 64)
    word1 &= (1 << 64) - 1
    carry = (tl + word1) >> 64
    quotient = th + word2 + carry
    assert quotient <= tp // q <= quotient + 3
    c = tp - quotient * q
    corrections = 0
    while c >= q:
        c -= q
        corrections += 1
    assert corrections <= 3
    return c


def multiply(plan: Plan, a: list, b: list) -> list:
    """Full pipeline for Python-int coefficient lists a, b (canonical, < q)."""
    return stages(plan, a, b)["c"]


def stages(plan: Plan, a: list, b: list) -> dict:
    """Intermediate buffers of the pipeline: v[k][i] (CRT inputs), dots[i][w], c[i]."""
    n, s, ns = plan.n, plan.split, plan.n_sub
    big_p, weights, rneg, finish = crt_constants(plan)
    r = len(plan.primes)
    residues = [[0] * n for _ in range(r)]  # v_k in natural coefficient order
    for k, p in enumerate(plan.primes):
        fwd, inv, zeta = twiddles(plan, k)
        spec_a = [ntt_forward([convert(plan, a[s * j + t], k) for j in range(ns)], fwd, p) for t in range(s)]
        spec_b = [ntt_forward([convert(plan, b[s * j + t], k) for j in range(ns)], fwd, p) for t in range(s)]
        for v in range(s):
            col = []
            for m in range(ns):
                low = sum(mont(spec_a[t][m], spec_b[v - t][m], p) for t in range(v + 1)) % p
                wrap = sum(mont(spec_a[t][m], spec_b[v + s - t][m], p) for t in range(v + 1, s)) % p
                col.append((low + shoup(wrap, zeta[m], p)) % p)
            out = ntt_inverse(col, inv, p)
            for j in range(ns):
                residues[k][s * j + v] = shoup(out[j], finish[k], p)
    words = plan.limbs + 5
    result, all_dots = [], []
    for i in range(n):
        # byte-sliced CRT: G[c] over byte columns, grouped into u64 word sums
        cols = [0] * (4 * words + 3)
        for k in range(r):
            vk = residues[k][i]
            for d in range(4):
                bd = byte(vk, d)
                if bd:
                    for c in range(d, 4 * words + 3):
                        cols[c] += bd * byte(weights[k], c - d)
        assert all(c < (1 << 31) for c in cols)
        dots = [sum(cols[4 * w + d] << (8 * d) for d in range(4) if 4 * w + d < len(cols)) for w in range(words + 1)]
        all_dots.append(dots[:words])
        result.append(reduce_words(plan, dots, rneg))
    return {"v": residues, "dots": all_dots, "c": result}


def schoolbook(a: list, b: list, q: int) -> list:
    n = len(a)
    out = [0] * n
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            k = i + j
            if k < n:
                out[k] += x * y
            else:
                out[k - n] -= x * y
    return [v % q for v in out]
