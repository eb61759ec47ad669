// Parameter-only plan: primes, roots of unity and exact CRT constants.
//
// Follows the reference's init (candidates/ordered-streaming/solve.cu:900-999):
// primes p = 1 (mod 2N') in [2^30, 2^31) scanned downward from 2^31 until
// P > 4N(q-1)^2 (:906-913), Miller-Rabin primality (src/big_unsigned.h:70-87),
// CRT partials P/p_k (mod q) (:944-949), psi search (:951), finish factors
// folding N'^-1 (P/p_k)^-1 (:953). Differences, by design:
//  * the ring is split s ways (N' = N/s) so that enough primes exist at
//    large N and L (the reference throws "insufficient independent NTT
//    fields" there, :910);
//  * M_k = (P/p_k) mod q is obtained in O(L) per prime by an exact division
//    ((P mod q) + m q) / p_k instead of a long division of P/p_k by q;
//  * any q >= 2 is supported: the final reduction is a Barrett step on the
//    top 64 bits of q (constants q_top, mu_low), not the reference's
//    q = 2^W - gap fold (src/solve.cu:448-467).
#include "host_plan.h"

#include <algorithm>
#include <thread>

namespace negacyclic {
namespace {

using Big = std::vector<uint32_t>;
using u128 = unsigned __int128;

void trim(Big& a) {
    while (a.size() > 1 && a.back() == 0) a.pop_back();
}

uint32_t bit_length(const Big& a) {
    for (size_t i = a.size(); i-- > 0;)
        if (a[i]) return uint32_t(i * 32 + 32 - __builtin_clz(a[i]));
    return 0;
}

int compare(const Big& a, const Big& b) {
    size_t n = std::max(a.size(), b.size());
    for (size_t i = n; i-- > 0;) {
        uint32_t x = i < a.size() ? a[i] : 0, y = i < b.size() ? b[i] : 0;
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

// a -= b, requires a >= b
void subtract_in_place(Big& a, const Big& b) {
    uint64_t borrow = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        uint64_t t = (i < b.size() ? uint64_t(b[i]) : 0) + borrow;
        uint32_t before = a[i];
        a[i] = before - uint32_t(t);
        borrow = (t >> 32) + (before < uint32_t(t) ? 1 : 0);
    }
    trim(a);
}

Big multiply_word(const Big& a, uint32_t w) {
    Big out(a.size() + 1, 0);
    uint64_t carry = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        uint64_t t = uint64_t(a[i]) * w + carry;
        out[i] = uint32_t(t);
        carry = t >> 32;
    }
    out[a.size()] = uint32_t(carry);
    trim(out);
    return out;
}

Big add(const Big& a, const Big& b) {
    Big out(std::max(a.size(), b.size()) + 1, 0);
    uint64_t carry = 0;
    for (size_t i = 0; i + 1 < out.size(); ++i) {
        uint64_t t = uint64_t(i < a.size() ? a[i] : 0) + (i < b.size() ? b[i] : 0) + carry;
        out[i] = uint32_t(t);
        carry = t >> 32;
    }
    out.back() = uint32_t(carry);
    trim(out);
    return out;
}

Big multiply(const Big& a, const Big& b) {
    Big out(a.size() + b.size(), 0);
    for (size_t i = 0; i < a.size(); ++i) {
        uint64_t carry = 0;
        for (size_t j = 0; j < b.size(); ++j) {
            uint64_t t = uint64_t(a[i]) * b[j] + out[i + j] + carry;
            out[i + j] = uint32_t(t);
            carry = t >> 32;
        }
        out[i + b.size()] = uint32_t(carry);
    }
    trim(out);
    return out;
}

uint32_t mod_word(const Big& a, uint32_t p) {
    uint64_t rem = 0;
    for (size_t i = a.size(); i-- > 0;) rem = ((rem << 32) | a[i]) % p;
    return uint32_t(rem);
}

// a / p for a divisible by p
Big divide_exact_word(const Big& a, uint32_t p) {
    Big out(a.size(), 0);
    uint64_t rem = 0;
    for (size_t i = a.size(); i-- > 0;) {
        uint64_t t = (rem << 32) | a[i];
        out[i] = uint32_t(t / p);
        rem = t % p;
    }
    trim(out);
    return out;
}

// Bits [at, at+32) of a; positions below 0 or above the top read as zero.
uint32_t word_at(const Big& a, int64_t at) {
    int64_t w = at >= 0 ? at / 32 : -((-at + 31) / 32);  // floor(at / 32)
    int64_t offset = at - w * 32;                        // 0..31
    uint64_t lo = (w >= 0 && w < int64_t(a.size())) ? a[size_t(w)] : 0;
    uint64_t hi = (w + 1 >= 0 && w + 1 < int64_t(a.size())) ? a[size_t(w + 1)] : 0;
    return uint32_t(((hi << 32) | lo) >> offset);
}

// 128 bits of a starting at bit `shift` (shift may be negative: low bits are zero).
u128 bits_at(const Big& a, int64_t shift) {
    u128 out = 0;
    for (int c = 0; c < 4; ++c) out |= u128(word_at(a, shift + 32 * c)) << (32 * c);
    return out;
}

struct Modulus {
    Big q;
    uint32_t bits = 0;
    int32_t shift = 0;  // bits - 64
    uint64_t top = 0;   // floor(q / 2^shift), in [2^63, 2^64)
};

// x mod q for x < q * 2^64, by one quotient estimate on the top bits.
Big reduce(const Big& x, const Modulus& m) {
    u128 top = bits_at(x, m.shift);
    u128 divisor = u128(m.top) + 1;
    uint64_t estimate = uint64_t(top / divisor);
    Big rem = x;
    if (estimate) {
        Big product = multiply(m.q, Big{uint32_t(estimate), uint32_t(estimate >> 32)});
        subtract_in_place(rem, product);
    }
    int guard = 0;
    while (compare(rem, m.q) >= 0) {
        subtract_in_place(rem, m.q);
        if (++guard > 4) break;
    }
    return rem;
}

uint32_t power_mod(uint64_t a, uint64_t e, uint32_t p) {
    uint64_t out = 1 % p;
    a %= p;
    for (; e; e >>= 1, a = a * a % p)
        if (e & 1) out = out * a % p;
    return uint32_t(out);
}

bool is_prime(uint32_t n) {
    if (n < 2) return false;
    for (uint32_t p : {2u, 3u, 5u, 7u})
        if (n % p == 0) return n == p;
    uint32_t d = n - 1, s = 0;
    while (!(d & 1)) {
        d >>= 1;
        ++s;
    }
    // bases {2,3,5,7} are deterministic below 3,215,031,751
    for (uint32_t a : {2u, 3u, 5u, 7u}) {
        uint64_t x = power_mod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (uint32_t j = 1; j < s; ++j) {
            x = x * x % n;
            if (x == n - 1) {
                composite = false;
                break;
            }
        }
        if (composite) return false;
    }
    return true;
}

// Primes p = 1 mod 2*n_sub, p in [2^30, 2^31), p not dividing q, until the
// product exceeds `bound`. Empty result when the range runs out.
std::vector<uint32_t> select_primes(uint32_t n_sub, const Big& q, const Big& bound) {
    std::vector<uint32_t> primes;
    Big product{1};
    uint64_t step = 2 * uint64_t(n_sub);
    uint64_t candidate = (uint64_t(kPrimeHigh) - 2) / step * step + 1;
    while (compare(product, bound) <= 0) {
        if (candidate < kPrimeLow) return {};
        uint32_t p = uint32_t(candidate);
        if (is_prime(p) && mod_word(q, p) != 0) {
            primes.push_back(p);
            product = multiply_word(product, p);
        }
        candidate -= step;
    }
    return primes;
}

uint32_t inverse_mod(uint32_t a, uint32_t p) { return power_mod(a, p - 2, p); }

}  // namespace

bool build_host_plan(uint32_t n, uint32_t limbs, const uint32_t* q_words, uint32_t requested_split,
                     HostPlan& plan, std::string& error, int& status) {
    status = 1;  // NEGACYCLIC_EINVAL
    if (n == 0 || (n & (n - 1)) || n > kMaxN) {
        error = "N must be a power of two in [1, " + std::to_string(kMaxN) + "]";
        return false;
    }
    if (limbs == 0 || limbs > 8000 || !q_words) {
        error = "L must be in [1, 8000] with q given";
        return false;
    }
    if (requested_split && ((requested_split & (requested_split - 1)) || requested_split > n ||
                            requested_split > kMaxSplit || n / requested_split > kMaxTransform)) {
        error = "split must be a power of two <= 16 with N/split <= 8192";
        return false;
    }
    Modulus m;
    m.q.assign(q_words, q_words + limbs);
    trim(m.q);
    m.bits = bit_length(m.q);
    if (m.bits < 2) {
        error = "q must be at least 2";
        return false;
    }
    m.shift = int32_t(m.bits) - 64;
    m.top = uint64_t(bits_at(m.q, m.shift));

    // bound = 4 N (q-1)^2 (candidates/ordered-streaming/solve.cu:906)
    Big q_minus_one = m.q;
    subtract_in_place(q_minus_one, Big{1});
    Big bound = multiply_word(multiply_word(multiply(q_minus_one, q_minus_one), n), 4);

    uint32_t split = requested_split ? requested_split : std::max<uint32_t>(1, n / kMaxTransform);
    std::vector<uint32_t> primes;
    for (;;) {
        primes = select_primes(n / split, m.q, bound);
        if (!primes.empty() || requested_split) break;
        split *= 2;
        if (split > kMaxSplit || split > n) break;
    }
    if (primes.empty()) {
        status = 2;  // NEGACYCLIC_ENOFIELDS
        error = "insufficient independent NTT fields for this point";
        return false;
    }
    const uint32_t r = uint32_t(primes.size());
    // K-dimension bound of the CRT GEMM: 4 r' * 255^2 < 2^31 (int32 accumulators)
    if ((r + 31) / 32 * 32 * 4 > 33024 || (limbs + 3) / 4 * 4 * 4 > 33024) {
        error = "point too wide for exact int32 byte accumulation";
        return false;
    }

    plan.n = n;
    plan.limbs = limbs;
    plan.split = split;
    plan.n_sub = n / split;
    plan.q = Big(q_words, q_words + limbs);
    plan.q_bits = m.bits;
    plan.words = limbs + 5;
    plan.top_shift = m.shift;
    plan.q_top = m.top;
    if (m.top == ~uint64_t(0)) {
        plan.mu_low = 0;  // floor(2^128 / 2^64) - 2^64
    } else {
        u128 mu = (~u128(0)) / (u128(m.top) + 1);  // == floor(2^128 / (top+1)) since top+1 < 2^64 is not a power of two
        plan.mu_low = uint64_t(mu - (u128(1) << 64));
    }

    // P mod q, incrementally: P~ <- P~ * p_k mod q
    Big p_mod_q{1};  // q >= 2
    for (uint32_t p : primes) p_mod_q = reduce(multiply_word(p_mod_q, p), m);

    plan.primes.assign(r, PrimeInfo{});
    plan.crt_weights.assign(size_t(r) * plan.words, 0);
    const uint32_t n_sub = plan.n_sub;

    auto work = [&](uint32_t begin, uint32_t end) {
        for (uint32_t k = begin; k < end; ++k) {
            const uint32_t p = primes[k];
            PrimeInfo& info = plan.primes[k];
            info.p = p;
            uint32_t inv = 1;  // p^-1 mod 2^32 by Newton iteration
            for (int i = 0; i < 5; ++i) inv *= 2 - p * inv;
            info.pinv = 0u - inv;
            const uint32_t radix = uint32_t((uint64_t(1) << 32) % p);
            info.r2 = uint32_t(uint64_t(radix) * radix % p);
            // (P/p_k) mod p_k = prod_{j != k} p_j mod p_k
            uint64_t partial = 1;
            for (uint32_t j = 0; j < r; ++j)
                if (j != k) partial = partial * (primes[j] % p) % p;
            uint64_t finish = uint64_t(info.r2) * radix % p;            // 2^96
            finish = finish * inverse_mod(n_sub % p, p) % p;            // N'^-1
            finish = finish * inverse_mod(uint32_t(partial), p) % p;    // (P/p_k)^-1
            info.finish = uint32_t(finish);
            info.finish_q = uint32_t((finish << 32) / p);
            // psi: g^((p-1)/2N') for a quadratic non-residue g
            uint32_t g = 2;
            while (power_mod(g, (p - 1) / 2, p) != p - 1) ++g;
            info.psi = power_mod(g, (p - 1) / (2 * uint64_t(n_sub)), p);
            // M_k = (P/p_k) mod q = ((P mod q) + m q) / p_k (mod q), m = -(P mod q) q^-1 mod p_k
            uint32_t pm = mod_word(p_mod_q, p), qm = mod_word(m.q, p);
            uint32_t mult = uint32_t((uint64_t(p - pm) % p) * inverse_mod(qm, p) % p);
            Big x = add(p_mod_q, multiply_word(m.q, mult));
            Big mk = divide_exact_word(x, p);
            if (compare(mk, m.q) >= 0) subtract_in_place(mk, m.q);
            uint32_t* row = &plan.crt_weights[size_t(k) * plan.words];
            for (size_t w = 0; w < mk.size() && w < limbs; ++w) row[w] = mk[w];
            const uint64_t f = ~uint64_t(0) / p;  // floor(2^64 / p) for odd p
            row[limbs + 2] = uint32_t(f);
            row[limbs + 3] = uint32_t(f >> 32);
        }
    };
    const uint32_t threads = std::max(1u, std::min<uint32_t>(std::thread::hardware_concurrency(), (r + 63) / 64));
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t)
        pool.emplace_back(work, uint32_t(uint64_t(r) * t / threads), uint32_t(uint64_t(r) * (t + 1) / threads));
    for (auto& th : pool) th.join();

    plan.minus_p_mod_q.assign(limbs, 0);
    if (!(p_mod_q.size() == 1 && p_mod_q[0] == 0)) {
        Big neg = m.q;
        subtract_in_place(neg, p_mod_q);
        for (size_t w = 0; w < neg.size() && w < limbs; ++w) plan.minus_p_mod_q[w] = neg[w];
    }
    status = 0;
    return true;
}

}  // namespace negacyclic
