// Host-side parameter plan for the negacyclic product (parameter-only, no
// operand data). Replaces the reference's init-time selection
// (candidates/ordered-streaming/solve.cu:900-999, src/big_unsigned.h).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace negacyclic {

constexpr uint32_t kPrimeLow = 1u << 30;
constexpr uint32_t kPrimeHigh = 1u << 31;
constexpr uint32_t kMaxTransform = 8192;  // N' = N / s <= 8192: one transform per CTA
constexpr uint32_t kMaxSplit = 16;
constexpr uint32_t kMaxN = kMaxTransform * kMaxSplit;

struct PrimeInfo {
    uint32_t p;
    uint32_t pinv;      // -p^-1 mod 2^32 (additive Montgomery reduction)
    uint32_t finish;    // 2^96 * N'^-1 * (P/p)^-1 mod p
    uint32_t finish_q;  // floor(finish * 2^32 / p)  (Shoup)
    uint32_t psi;       // primitive 2N'-th root of unity
    uint32_t r2;        // 2^64 mod p (to enter Montgomery form)
};

struct HostPlan {
    uint32_t n = 0, limbs = 0, split = 1, n_sub = 1, q_bits = 0;
    std::vector<uint32_t> q;              // limbs words
    std::vector<PrimeInfo> primes;        // r
    std::vector<uint32_t> crt_weights;    // [r][words]: W_k = M_k + 2^(32(L+2)) * floor(2^64/p_k)
    std::vector<uint32_t> minus_p_mod_q;  // [limbs]: (-P) mod q
    uint32_t words = 0;                   // L + 5
    // Barrett constants of the final reduction: q_top = top 64 bits of q
    // (q shifted so bit 63 is its top bit), mu = floor(2^128 / (q_top + 1)) - 2^64.
    int32_t top_shift = 0;                // bitlen(q) - 64 (may be negative)
    uint64_t q_top = 0, mu_low = 0;
};

// Builds the plan. Returns false with `error` set when the point is invalid or
// no split up to kMaxSplit has enough primes. `requested_split` 0 = automatic.
bool build_host_plan(uint32_t n, uint32_t limbs, const uint32_t* q, uint32_t requested_split,
                     HostPlan& plan, std::string& error, int& status);

}  // namespace negacyclic
