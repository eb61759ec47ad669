// 31-bit prime-field arithmetic used by every kernel (p in [2^30, 2^31)).
//
// Same exactness conditions as the reference's helpers
// (src/solve.cu:39-52; proofs in candidates/pipelined-direct-crt/EXACTNESS.md:59-66
// and candidates/ordered-streaming/README.md:42-47), written here as:
//  * redc: additive Montgomery reduction, t < p 2^32 -> t 2^-32 mod p;
//  * shoup: a w mod p with a precomputed w' = floor(w 2^32 / p), any a < 2^32.
#pragma once
#include <cstdint>

namespace negacyclic {

struct DevicePrime {
    uint32_t p;
    uint32_t pinv;      // -p^-1 mod 2^32
    uint32_t finish;    // 2^96 N'^-1 (P/p)^-1 mod p
    uint32_t finish_q;  // Shoup quotient of finish
    uint32_t psi;       // primitive 2N'-th root
    uint32_t r2;        // 2^64 mod p
};

// Conditional subtractions as unsigned minima: for t in [0, 2p) with 2p < 2^32,
// t - p wraps above t exactly when t < p, so min(t, t - p) is t mod p.
__device__ __forceinline__ uint32_t reduce_once(uint32_t t, uint32_t p) { return min(t, t - p); }

__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) { return reduce_once(a + b, p); }

// a, b in [0, p): a - b wraps when a < b, and then a - b + p is the smaller value
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
    const uint32_t t = a - b;
    return min(t, t + p);
}

// t < p * 2^32  ->  t * 2^-32 mod p, canonical
__device__ __forceinline__ uint32_t redc(uint64_t t, uint32_t p, uint32_t pinv) {
    uint32_t m = uint32_t(t) * pinv;
    uint32_t u = uint32_t((t + uint64_t(m) * p) >> 32);
    return reduce_once(u, p);
}

__device__ __forceinline__ uint32_t mont(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    return redc(uint64_t(a) * b, p, pinv);
}

// a * w mod p, w < p, w_q = floor(w 2^32 / p), any 32-bit a
__device__ __forceinline__ uint32_t shoup(uint32_t a, uint32_t w, uint32_t w_q, uint32_t p) {
    uint32_t quotient = __umulhi(a, w_q);
    uint32_t r = a * w - quotient * p;
    return reduce_once(r, p);
}

// base^e mod p in standard form, via Montgomery squaring
__device__ __forceinline__ uint32_t pow_mod(uint32_t base, uint64_t e, const DevicePrime& f) {
    uint32_t x = mont(base % f.p, f.r2, f.p, f.pinv);  // base * 2^32
    uint32_t acc = mont(1, f.r2, f.p, f.pinv);          // 2^32 (Montgomery one)
    for (; e; e >>= 1) {
        if (e & 1) acc = mont(acc, x, f.p, f.pinv);
        x = mont(x, x, f.p, f.pinv);
    }
    return mont(acc, 1, f.p, f.pinv);
}

// shoup without its final correction: a w mod p + {0 or p}, in [0, 2p) for any 32-bit a
// (the quotient estimate is at most one short; Harvey, "Faster arithmetic for number-theoretic
// transforms", J. Symb. Comput. 60 (2014), lemma on Shoup's multiplication)
__device__ __forceinline__ uint32_t shoup_lazy(uint32_t a, uint32_t w, uint32_t w_q, uint32_t p) {
    return a * w - __umulhi(a, w_q) * p;
}

__device__ __forceinline__ uint32_t shoup_quotient(uint32_t w, uint32_t p) {
    return uint32_t((uint64_t(w) << 32) / p);
}

}  // namespace negacyclic
