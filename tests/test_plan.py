"""Host plan and pipeline algebra (no GPU).

* the exact model of the device pipeline (tests/model.py) equals a schoolbook
  product, for every ring split, including extremal operands;
* the library's host plan (primes, split, finish factors, M_k = (P/p_k) mod q,
  (-P) mod q) equals the model's independent Python computation;
* the arithmetic identities the kernels rely on, at the new parameters:
  fixed-point CRT quotient, shortened CRT, byte-sum and REDC bounds, and the
  final Barrett step (ports of the reference's tests/direct_crt_math.py and
  tests/tensor_montgomery_math.py).
"""
import random

import numpy as np
import pytest

import model


@pytest.mark.parametrize("n,limbs,split", [(1, 1, None), (2, 1, None), (4, 2, None), (8, 3, 2), (16, 2, 4),
                                           (16, 4, 16), (32, 5, None), (64, 2, 8)])
def test_model_matches_schoolbook(n, limbs, split):
    rng = random.Random(n * 131 + limbs)
    for trial in range(3):
        q = rng.randrange(1 << (32 * limbs - 32), 1 << (32 * limbs)) | 1
        q = max(q, 3)
        if trial == 0:
            a = [rng.randrange(q) for _ in range(n)]
            b = [rng.randrange(q) for _ in range(n)]
        elif trial == 1:
            a, b = [q - 1] * n, [q - 1] * n
        else:
            a, b = [0] * n, [q - 1] * n
            a[0] = 1
        plan = model.make_plan(n, limbs, q, split)
        assert model.multiply(plan, a, b) == model.schoolbook(a, b, q)


POINTS = [(1, 1, 0x3), (64, 1, 0xFFFFFFFB), (4096, 64, None), (8192, 8, None), (32768, 28, None),
          (65536, 55, None), (131072, 4, None)]


@pytest.mark.parametrize("n,limbs,qv", POINTS)
def test_host_plan_matches_model(n, limbs, qv, fpc, inputs):
    q_arr = inputs.random_modulus(limbs, n + limbs) if qv is None else inputs.from_int(qv, limbs)
    q = inputs.to_int(q_arr)
    host = fpc.host_plan(n, limbs, q_arr)
    ref = model.make_plan(n, limbs, q)
    assert host["split"] == ref.split and host["n_sub"] == ref.n_sub
    assert list(host["primes"]) == ref.primes
    big_p, weights, rneg, finish = model.crt_constants(ref)
    assert list(host["finish"]) == finish
    mask = (1 << (32 * (limbs + 2))) - 1
    for k in (0, len(ref.primes) // 2, len(ref.primes) - 1):
        assert inputs.to_int(host["crt_mod_q"][k]) == weights[k] & mask
    assert inputs.to_int(host["minus_p_mod_q"]) == rneg
    assert big_p > 4 * n * (q - 1) ** 2


def test_host_plan_at_full_size_configs(fpc, inputs):
    # the three sizes the benchmark and parity runs use: enough primes after the split
    for n, limbs, seed, split in [(4096, 64, 0, 1), (32768, 868, 1, 4), (65536, 1747, 2, 8)]:
        q = inputs.random_modulus(limbs, seed)
        host = fpc.host_plan(n, limbs, q)
        assert host["split"] == split
        primes = [int(p) for p in host["primes"]]
        assert all((1 << 30) <= p < (1 << 31) and (p - 1) % (2 * host["n_sub"]) == 0 for p in primes)
        assert len(set(primes)) == len(primes)
        assert sum(np.log2(primes)) > np.log2(4 * n) + 2 * (32 * limbs)  # P > 4N(q-1)^2


def test_host_plan_rejects_invalid_points(fpc):
    q = np.array([7], np.uint32)
    for n in (0, 3, 1 << 18):
        with pytest.raises(RuntimeError):
            fpc.host_plan(n, 1, q)
    with pytest.raises(RuntimeError):
        fpc.host_plan(16, 1, np.array([1], np.uint32))  # q < 2
    with pytest.raises(RuntimeError):
        fpc.host_plan(16, 1, q, split=3)


@pytest.mark.parametrize("n,limbs", [(128, 4), (8192, 8), (32768, 28), (65536, 55), (4096, 64)])
def test_fixed_point_crt_quotient_and_shortened_crt(n, limbs):
    """tests/direct_crt_math.py restated for the split-ring primes and appended-weight quotient."""
    rng = random.Random(0xC47 + n + limbs)
    q = rng.randrange(1 << (32 * limbs - 32), 1 << (32 * limbs)) | 1
    plan = model.make_plan(n, limbs, q)
    big_p, weights, rneg, finish = model.crt_constants(plan)
    primes = plan.primes
    partial = [big_p // p for p in primes]
    inv = [pow(m, -1, p) for m, p in zip(partial, primes)]
    f = [(1 << 64) // p for p in primes]
    mk = [m % q for m in partial]
    bound = n * (q - 1) ** 2
    values = [-bound, -bound + 1, -q, -q + 1, -1, 0, 1, q - 1, q, bound - 1, bound]
    values += [rng.randrange(-bound, bound + 1) for _ in range(200)]
    for x in values:
        v = [(x % p) * a % p for p, a in zip(primes, inv)]
        true_k = (sum(a * b for a, b in zip(v, partial)) - x) // big_p
        d = sum(a * b for a, b in zip(v, f))
        assert (d + (1 << 63)) >> 64 == true_k
        t = sum(a * b for a, b in zip(v, mk))
        assert t < 1 << (32 * (limbs + 2))
        assert d < 1 << 96
        assert (t + true_k * rneg) % q == x % q
        assert (t + true_k * rneg) // q < 1 << 48


def test_byte_sum_and_redc_bounds():
    """tests/tensor_montgomery_math.py restated: u8 dot products stay exact in int32; REDC is canonical."""
    for k_bytes in (4 * 1748, 4 * 3648, 33024):
        assert k_bytes * 255 * 255 < 1 << 31
    max_sum = 33024 * 255 * 255 * sum(1 << (8 * i) for i in range(4))
    assert max_sum < 1 << 56 and max_sum < (1 << 30) << 32  # REDC needs S < p 2^32
    rng = random.Random(20261110)
    for p in [(1 << 30) + 1, 2147352577] + [rng.randrange(1 << 29, 1 << 30) * 2 + 1 for _ in range(30)]:
        for value in [0, 1, p - 1, p, max_sum] + [rng.randrange(max_sum + 1) for _ in range(30)]:
            assert model.redc(value, p) == value * pow(1 << 32, -1, p) % p


def test_barrett_reduce_step_bounds():
    """The reduce kernel's single quotient step leaves at most three subtractions."""
    rng = random.Random(99)
    for limbs in (1, 2, 3, 55, 64):
        q = rng.randrange(1 << (32 * limbs - 32), 1 << (32 * limbs)) | 1
        q = max(q, 3)
        plan = model.Plan(1, limbs, q, 1, 1, [])
        for _ in range(50):
            tp = rng.randrange(0, q << 47)
            dots = [(tp >> (32 * w)) & 0xFFFFFFFF for w in range(limbs + 5)]
            assert model.reduce_words(plan, dots, 0) == tp % q


M32, M64 = (1 << 32) - 1, (1 << 64) - 1


def _chain_carry(generate, propagate, chain):
    """chain_carry in kernels.cu: carries into 32 lanes from generate/propagate ballots."""
    g = sum(1 << lane for lane in range(32) if generate[lane])
    gp = g | sum(1 << lane for lane in range(32) if propagate[lane])
    full = gp + g + chain
    carries = (full ^ gp ^ g) & M32
    return [(carries >> lane) & 1 for lane in range(32)], full >> 32


def _reduce_add_pass(d, r_words, k, tlen):
    """Step 2 of reduce_kernel: T' words from word sums d[w] + K R[w], two words per lane."""
    limbs, v = len(r_words), [0] * tlen
    chain = carried_high = 0
    for base in range(0, tlen, 64):
        x0, x1 = [], []
        for lane in range(32):
            w0 = base + 2 * lane
            x0.append((d[w0] if w0 < tlen else 0) + k * (r_words[w0] if w0 < limbs else 0))
            x1.append((d[w0 + 1] if w0 + 1 < tlen else 0) + k * (r_words[w0 + 1] if w0 + 1 < limbs else 0))
        top = [x >> 32 for x in x1]
        below, carried_high = [carried_high] + top[:31], top[31]
        generate, propagate, words = [], [], []
        for lane in range(32):
            s0 = (x0[lane] & M32) + below[lane]
            s1 = (x0[lane] >> 32) + (x1[lane] & M32) + (s0 >> 32)
            assert s0 < 1 << 33 and s1 < 1 << 33
            gen = (s1 >> 32) != 0
            generate.append(gen)
            propagate.append(not gen and (s0 & s1 & M32) == M32)
            words.append((s0 & M32, s1 & M32))
        carries, chain = _chain_carry(generate, propagate, chain)
        for lane in range(32):
            w0 = base + 2 * lane
            word0 = (words[lane][0] + carries[lane]) & M32
            word1 = (words[lane][1] + (1 if carries[lane] and word0 == 0 else 0)) & M32
            if w0 < tlen:
                v[w0] = word0
            if w0 + 1 < tlen:
                v[w0 + 1] = word1
    return v


def _reduce_sub_pass(v, q_words, quotient, tlen):
    """Step 4 of reduce_kernel: T' - quotient q with signed word carries, two words per lane."""
    limbs, out = len(q_words), [0] * tlen
    ql, qh = quotient & M32, quotient >> 32
    chain = carry_hi = carry_c = 0
    qw = lambda w: q_words[w] if 0 <= w < limbs else 0  # noqa: E731
    for base in range(0, tlen, 64):
        lanes = []
        for lane in range(32):
            w0 = base + 2 * lane
            a0, b0, a1, b1 = ql * qw(w0), qh * qw(w0 - 1), ql * qw(w0 + 1), qh * qw(w0)
            lanes.append((w0, a0, b0, a1, b1, (a0 >> 32) + (b0 >> 32), (a1 >> 32) + (b1 >> 32)))
        hi_below, carry_hi = [carry_hi] + [x[6] for x in lanes[:31]], lanes[31][6]
        zs = []
        for lane, (w0, a0, b0, a1, b1, hi0, _) in enumerate(lanes):
            e0 = (a0 & M32) + (b0 & M32) + hi_below[lane]
            e1 = (a1 & M32) + (b1 & M32) + hi0
            assert e0 < 1 << 35 and e1 < 1 << 35
            zs.append(((v[w0] if w0 < tlen else 0) - e0, (v[w0 + 1] if w0 + 1 < tlen else 0) - e1))
        c1 = [z1 >> 32 for _, z1 in zs]
        c_below, carry_c = [carry_c] + c1[:31], c1[31]
        generate, propagate, sws = [], [], []
        for lane, (z0, z1) in enumerate(zs):
            sw0, sw1 = (z0 & M32) + c_below[lane], (z1 & M32) + (z0 >> 32)
            assert -8 <= sw0 < 1 << 32 and -8 <= sw1 < 1 << 32
            gen = sw1 < 0 or (sw1 == 0 and sw0 < 0)
            generate.append(gen)
            propagate.append(not gen and sw1 == 0 and sw0 == 0)
            sws.append((sw0, sw1))
        borrows, chain = _chain_carry(generate, propagate, chain)
        for lane, (sw0, sw1) in enumerate(sws):
            w0, t0 = base + 2 * lane, sw0 - borrows[lane]
            if w0 < tlen:
                out[w0] = t0 & M32
            if w0 + 1 < tlen:
                out[w0 + 1] = (sw1 - (1 if t0 < 0 else 0)) & M32
    return out


def test_reduce_carry_passes_two_words_per_lane():
    """The reduce kernel's two carry passes, restated lane by lane (32 lanes, two adjacent words
    each, one ballot-based carry resolution per 64 words), against big-integer arithmetic. Runs
    of all-ones and zero words exercise carries and borrows that cross many lanes and steps."""
    rng = random.Random(2027)
    value = lambda words: sum(x << (32 * i) for i, x in enumerate(words))  # noqa: E731
    subtractions = 0
    for trial in range(400):
        limbs = rng.choice([1, 2, 31, 32, 33, 62, 63, 64, 65, 127, 129, 300])
        tlen, mode = limbs + 2, trial % 5
        sparse = mode == 4  # words from {0, 1, 2^32 - 1}: long zero and all-ones runs in T' and q
        pick = [lambda: rng.randrange(1 << 56), lambda: rng.choice([M32, (1 << 56) - 1]),
                lambda: rng.choice([0, 1 << 32]), lambda: rng.choice([0, M32, rng.randrange(1 << 56)]),
                lambda: rng.choice([0, 0, 0, 1, M32])][mode]
        d = [pick() for _ in range(tlen)]
        d[tlen - 1], d[tlen - 2] = 0, d[tlen - 2] & (M32 >> 8)  # T' stays below 2^(32 tlen)
        r_words = [rng.choice([0, 1, M32] if sparse else [0, M32, rng.randrange(1 << 32)]) for _ in range(limbs)]
        k = rng.choice([0, 1]) if sparse else rng.randrange(1 << 14)  # K < 2r
        exact = sum((d[w] + k * (r_words[w] if w < limbs else 0)) << (32 * w) for w in range(tlen))
        assert exact < 1 << (32 * tlen)
        v = _reduce_add_pass(d, r_words, k, tlen)
        assert value(v) == exact
        q_words = [rng.choice([0, 0, 1, M32] if sparse else [M32, 0, rng.randrange(1 << 32)]) for _ in range(limbs)]
        q_words[-1] = q_words[-1] or 1
        q = value(q_words)
        quotient = max(0, exact // q - rng.choice([0, 0, 1, 2, 3]))  # the Barrett step is at most 3 short
        if quotient >> 64:
            continue
        subtractions += 1
        assert value(_reduce_sub_pass(v, q_words, quotient, tlen)) == exact - quotient * q
    assert subtractions > 300
