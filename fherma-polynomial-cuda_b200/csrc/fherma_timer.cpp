// fherma_timer: times fherma_run the way the platform harness calls it (src/main.cpp:181-186),
// with operands generated in memory instead of read from case files.
//
//   fherma_timer N L SEED STEPS WARMUP
//
// The harness holds a, b and the returned c in pageable std::vectors, and fherma_run allocates
// a fresh output vector inside the timed call; so does this driver. q is a random odd L-limb
// value with a nonzero top limb, and every operand coefficient is below q (its top limb is
// below q's). Each timed call uses a different operand pair (STEPS + WARMUP pairs are kept in
// memory, so no call sees another call's data in a cache). Prints one JSON line with the
// per-call milliseconds (steady_clock around fherma_run alone, as the harness measures), and
// checks that a product and its operands swapped agree.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/fherma_b200.h"

namespace {

uint64_t splitmix(uint64_t& state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

fherma::Tensor<uint32_t> operand(uint32_t n, uint32_t limbs, const std::vector<uint32_t>& q, uint64_t seed) {
    fherma::Tensor<uint32_t> t;
    t.shape = {int64_t(n), int64_t(limbs)};
    t.data.resize(size_t(n) * limbs);
    uint64_t state = seed;
    for (size_t i = 0; i < t.data.size(); ++i) t.data[i] = uint32_t(splitmix(state));
    const uint32_t top = q[limbs - 1];  // >= 1: a top limb below it keeps the value below q
    for (size_t i = 0; i < n; ++i) t.data[i * limbs + limbs - 1] %= top;
    return t;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s N L SEED STEPS WARMUP\n", argv[0]);
        return 2;
    }
    const uint32_t n = uint32_t(std::atoi(argv[1])), limbs = uint32_t(std::atoi(argv[2]));
    const uint64_t seed = std::strtoull(argv[3], nullptr, 10);
    const int steps = std::atoi(argv[4]), warmup = std::atoi(argv[5]);
    if (!n || !limbs || steps < 1 || warmup < 0) return 2;
    uint64_t state = seed * 0x100000001B3ull + 1;
    fherma::Point point;
    point.N = n;
    point.W = 32 * limbs;
    point.L = limbs;
    point.q.shape = {int64_t(limbs)};
    point.q.data.resize(limbs);
    for (auto& w : point.q.data) w = uint32_t(splitmix(state));
    point.q.data[0] |= 1u;
    if (point.q.data[limbs - 1] == 0) point.q.data[limbs - 1] = 1;
    try {
        const auto t0 = std::chrono::steady_clock::now();
        void* handle = fherma_init(point);
        const double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::vector<fherma::Inputs> pairs(size_t(steps + warmup));
        for (size_t i = 0; i < pairs.size(); ++i) {
            pairs[i].a = operand(n, limbs, point.q.data, splitmix(state));
            pairs[i].b = operand(n, limbs, point.q.data, splitmix(state));
        }
        std::vector<double> ms;
        bool agree = true;
        for (size_t i = 0; i < pairs.size(); ++i) {
            const auto start = std::chrono::steady_clock::now();
            fherma::Outputs out = fherma_run(handle, pairs[i]);
            const auto stop = std::chrono::steady_clock::now();
            if (int(i) >= warmup) ms.push_back(std::chrono::duration<double, std::milli>(stop - start).count());
            if (i + 1 == pairs.size()) {  // a * b == b * a on the last pair
                fherma::Inputs swapped{pairs[i].b, pairs[i].a};
                agree = fherma_run(handle, swapped).c.data == out.c.data;
            }
        }
        fherma_free(handle);
        std::vector<double> sorted = ms;
        std::sort(sorted.begin(), sorted.end());
        double sum = 0;
        for (double x : ms) sum += x;
        std::printf(
            "{\"n\": %u, \"limbs\": %u, \"init_s\": %.3f, \"steps\": %d, \"median_ms\": %.4f, \"mean_ms\": %.4f, "
            "\"min_ms\": %.4f, \"max_ms\": %.4f, \"commutes\": %s}\n",
            n, limbs, init_s, steps, sorted[sorted.size() / 2], sum / ms.size(), sorted.front(), sorted.back(),
            agree ? "true" : "false");
        return agree ? 0 : 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "fherma_timer: %s\n", e.what());
        return 1;
    }
}
