// CPU check of the host path's copy team (fherma-polynomial-cuda_b200/csrc/host_io.h), built and
// run by tests/test_host_team.py: a pack job that publishes per-chunk counters while a launcher
// thread consumes chunks in order, an unpack job that follows per-chunk "landed" flags, blocking
// copies and touches, and many calls in a row with idle gaps (with a short spin, workers going to
// sleep and waking), stage_copy against memcpy, and that a team whose workers are spinning is
// destroyed at once.
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <thread>
#include <vector>

#include "../../fherma-polynomial-cuda_b200/csrc/host_io.h"

using negacyclic::HostTeam;

static int failures = 0;
#define EXPECT(cond)                                                          \
    do {                                                                      \
        if (!(cond)) {                                                        \
            std::fprintf(stderr, "%s:%d: %s\n", __FILE__, __LINE__, #cond);   \
            ++failures;                                                       \
        }                                                                     \
    } while (0)

static void run_calls(HostTeam& team, uint64_t seed) {
    std::mt19937_64 rng(seed);
    constexpr uint32_t kChunks = 16;
    for (int call = 0; call < 300; ++call) {
        const uint32_t limbs = 1 + uint32_t(rng() % 70), split = 1u << (rng() % 4);
        const uint32_t n_sub = 64 + uint32_t(rng() % 4) * 32, n = n_sub * split, chunks = std::min(kChunks, split * 2);
        std::vector<uint32_t> src(size_t(n) * limbs), stage(src.size(), 0u), out(src.size(), 0u);
        for (auto& x : src) x = uint32_t(rng());
        // input: chunk k = transform t, positions [j0, j0 + span): rows s*j + t -> t*N' + j
        std::atomic<uint32_t> packed[kChunks] = {};
        const uint32_t per_t = chunks / split ? chunks / split : 1, span = n_sub / per_t;
        std::vector<std::pair<uint32_t, uint32_t>> list;  // (t, j0)
        for (uint32_t t = 0; t < split; ++t)
            for (uint32_t j0 = 0; j0 < n_sub; j0 += span) list.emplace_back(t, j0);
        const uint64_t ticket = team.post([&, list](unsigned w, unsigned count) {
            for (uint32_t k = 0; k < list.size(); ++k) {
                const auto [t, j0] = list[k];
                const size_t first = HostTeam::slice_begin(span, w, count), last = HostTeam::slice_begin(span, w + 1, count);
                for (size_t j = first; j < last; ++j)
                    std::memcpy(&stage[(size_t(t) * n_sub + j0 + j) * limbs], &src[(size_t(split) * (j0 + j) + t) * limbs],
                                limbs * 4);
                packed[k].fetch_add(1, std::memory_order_release);
            }
        });
        for (uint32_t k = 0; k < list.size(); ++k) {  // the launcher: chunk k complete before use
            negacyclic::spin_until(packed[k], team.workers());
            const auto [t, j0] = list[k];
            for (uint32_t j = j0; j < j0 + span; ++j)
                EXPECT(std::memcmp(&stage[(size_t(t) * n_sub + j) * limbs], &src[(size_t(split) * j + t) * limbs],
                                   limbs * 4) == 0);
        }
        team.wait(ticket);
        // output: the team copies chunk k once this thread marks it landed
        std::atomic<uint32_t> landed[kChunks] = {};
        const uint32_t out_chunks = 1 + uint32_t(rng() % kChunks), per = (n + out_chunks - 1) / out_chunks;
        const uint64_t unpack = team.post([&](unsigned w, unsigned count) {
            for (uint32_t k = 0; k < out_chunks; ++k) {
                negacyclic::spin_until(landed[k], 1);
                const size_t first = size_t(k) * per, rows = first < n ? std::min<size_t>(per, n - first) : 0;
                const size_t words = rows * limbs, b = HostTeam::slice_begin(words, w, count),
                             e = HostTeam::slice_begin(words, w + 1, count);
                if (e > b) std::memcpy(&out[first * limbs + b], &src[first * limbs + b], (e - b) * 4);
            }
        });
        for (uint32_t k = 0; k < out_chunks; ++k) {
            if (rng() % 8 == 0) std::this_thread::sleep_for(std::chrono::microseconds(50));
            landed[k].store(1, std::memory_order_release);
        }
        team.wait(unpack);
        EXPECT(out == src);
        // blocking helpers
        std::vector<uint32_t> copy(src.size(), 0u);
        team.copy(copy.data(), src.data(), src.size() * 4);
        EXPECT(copy == src);
        team.touch(copy.data(), copy.size() * 4);
        EXPECT(std::all_of(copy.begin(), copy.end(), [](uint32_t x) { return x == 0; }));
        if (call % 50 == 49) std::this_thread::sleep_for(std::chrono::milliseconds(20));  // past a short spin
    }
}

int main(int argc, char** argv) {
    const unsigned workers = argc > 1 ? unsigned(std::atoi(argv[1])) : 5;
    {
        HostTeam team(workers);  // default spin: the workers stay awake between calls
        run_calls(team, 7);
    }
    {
        HostTeam team(workers, std::chrono::microseconds(200));  // workers sleep in the idle gaps
        run_calls(team, 8);
    }
    {  // stage_copy (streaming stores where the CPU has AVX-512): every size and misalignment
        std::mt19937_64 rng(9);
        std::vector<unsigned char> src(1 << 16), dst(src.size() + 256);
        for (auto& x : src) x = static_cast<unsigned char>(rng());
        for (int trial = 0; trial < 2000; ++trial) {
            const size_t bytes = trial < 600 ? size_t(trial) : size_t(rng() % (src.size() - 128));
            const size_t s_off = rng() % 64, d_off = rng() % 128;
            std::fill(dst.begin(), dst.end(), 0xA5);
            negacyclic::stage_copy(dst.data() + d_off, src.data() + s_off, bytes);
            negacyclic::store_fence();
            EXPECT(std::memcmp(dst.data() + d_off, src.data() + s_off, bytes) == 0);
            EXPECT(std::all_of(dst.begin(), dst.begin() + d_off, [](unsigned char x) { return x == 0xA5; }));
            EXPECT(std::all_of(dst.begin() + d_off + bytes, dst.end(), [](unsigned char x) { return x == 0xA5; }));
        }
    }
    {  // destroying a team whose workers are spinning does not wait out their spin
        auto team = std::make_unique<HostTeam>(workers);
        std::vector<uint32_t> a(1 << 16, 1u), b(a.size(), 0u);
        team->copy(b.data(), a.data(), a.size() * 4);
        EXPECT(a == b);
        const auto start = std::chrono::steady_clock::now();
        team.reset();
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
        const double spin_ms = std::chrono::duration<double, std::milli>(HostTeam::kSpinTime).count();
        EXPECT(ms < 0.5 * spin_ms);
    }
    std::printf("host team check: %d failures\n", failures);
    return failures ? 1 : 0;
}
