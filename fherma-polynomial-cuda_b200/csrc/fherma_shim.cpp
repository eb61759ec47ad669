// fherma_init / fherma_run / fherma_free over the C ABI (include/negacyclic.h).
//
// Behaviour follows the reference's plugin (src/solve.cu:503-614):
//  * init validates the point (N a power of two, L == (W+31)/32) and builds
//    parameter-only state; no operand-dependent work (README.md:40);
//  * run checks operand sizes, returns a freshly allocated Outputs{c} of shape
//    {N, L} (built on a helper thread while the product runs), and finishes all
//    work before returning;
//  * failures throw std::runtime_error with the library's message.
// Compile with -DFHERMA_TYPES_DEFINED and the platform's fherma.h included
// first to use the generated types instead of include/fherma_b200.h's.
#include <malloc.h>
#include <sys/mman.h>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <algorithm>
#include <atomic>
#include <chrono>

#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fherma_b200.h"
#include "../../include/negacyclic.h"

namespace {

// Builds the output vector that fherma_run must return, on a thread of its own, while the
// calling thread packs the operands and launches the product. std::vector value-initialises
// its elements on one core, and fresh pages fault one 4 KB page at a time: 156-160 ms for the
// 458 MB result of N=65536, L=1747 on a B200 host. Reserving first and asking for transparent
// huge pages over the reserved range (when it spans at least kHugeBytes) cuts that to 54 ms.
// The hint applies from 4 MB up: behind the reference's harness it also helped the 14.4 MB result
// of N=65536, L=55 (see keep_heap_resident below for the measurement).
// After the fill the thread keeps spinning until the call is over (release(), or kActiveFor):
// on a B200 box's virtual host, copy threads writing lines that this thread had just zeroed,
// once it slept, took ~300 us for the last 1.8 MB output chunk instead of ~35, and the device's
// reads of host memory also slowed while host cores idled.
class OutputBuilder {
public:
    OutputBuilder() : thread_([this] { loop(); }) {}

    ~OutputBuilder() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
        }
        released_.store(true);
        cv_.notify_all();
        thread_.join();
    }

    void start(size_t count) {
        std::lock_guard<std::mutex> lock(mu_);
        count_ = count;
        ready_ = false;
        requested_ = true;
        released_.store(false);
        cv_.notify_all();
    }

    std::vector<uint32_t> take() {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return ready_; });
        ready_ = false;
        return std::move(built_);
    }

    // The call that started the build is over: the thread may stop spinning.
    void release() { released_.store(true); }

private:
    static constexpr size_t kHugeBytes = size_t(4) << 20;
    static constexpr std::chrono::milliseconds kActiveFor{50};

    static void build(std::vector<uint32_t>& v, size_t count) {
        v.reserve(count);
        const size_t bytes = count * sizeof(uint32_t);
        if (bytes >= kHugeBytes) {  // a hint only; small arrays fault fast enough without it
            const uintptr_t huge = uintptr_t(2) << 20;
            const uintptr_t begin = (reinterpret_cast<uintptr_t>(v.data()) + huge - 1) & ~(huge - 1);
            const uintptr_t end = (reinterpret_cast<uintptr_t>(v.data()) + bytes) & ~(huge - 1);
            if (end > begin) madvise(reinterpret_cast<void*>(begin), end - begin, MADV_HUGEPAGE);
        }
        v.resize(count);
    }

    void loop() {
        std::unique_lock<std::mutex> lock(mu_);
        for (;;) {
            cv_.wait(lock, [&] { return stop_ || requested_; });
            if (stop_) return;
            requested_ = false;
            const size_t count = count_;
            lock.unlock();
            std::vector<uint32_t> v;
            build(v, count);
            lock.lock();
            built_ = std::move(v);
            ready_ = true;
            cv_.notify_all();
            lock.unlock();
            const auto until = std::chrono::steady_clock::now() + kActiveFor;
            while (!released_.load(std::memory_order_acquire) && std::chrono::steady_clock::now() < until) pause();
            lock.lock();
        }
    }

    static void pause() {
#if defined(__x86_64__)
        _mm_pause();
#else
        std::this_thread::yield();
#endif
    }

    std::mutex mu_;
    std::condition_variable cv_;
    bool stop_ = false, requested_ = false, ready_ = false;
    std::atomic<bool> released_{true};
    size_t count_ = 0;
    std::vector<uint32_t> built_;
    std::thread thread_;
};

struct State {
    negacyclic_plan* plan = nullptr;
    uint32_t n = 0, limbs = 0;
    OutputBuilder output;
};

// The platform harness allocates the operands and the result of every case afresh and frees them
// after it. With glibc's defaults the freed heap top goes back to the operating system after each
// case, so every fherma_run faults the pages of its fresh result vector in again while filling it
// (one 4 KB page at a time on a virtual host). fherma_init therefore keeps freed heap memory in
// the process: arrays up to 32 MB come from the heap, and the heap top is trimmed only beyond
// 1 GB. Behind the reference's harness at N=65536, L=55 this took fherma_run from 1.69 to 1.45 ms
// together with the huge-page hint above (from 1.69 to 1.52 ms alone), and from 0.532 to 0.518 ms
// at N=32768, L=28 (medians of 20 cases, 4 alternating runs on one box). Set
// NEGACYCLIC_KEEP_MALLOC=1 to leave the process's allocator settings alone.
void keep_heap_resident() {
    const char* keep = std::getenv("NEGACYCLIC_KEEP_MALLOC");
    if (keep && *keep && *keep != '0') return;
    mallopt(M_MMAP_THRESHOLD, 32 << 20);
    mallopt(M_TRIM_THRESHOLD, 1 << 30);
}

[[noreturn]] void raise(const char* what) {
    throw std::runtime_error(std::string(what) + ": " + negacyclic_last_error());
}

}  // namespace

void* fherma_init(const fherma::Point& point) {
    if (point.q.data.size() != point.L) throw std::runtime_error("q must hold L words");
    keep_heap_resident();
    auto* state = new State;
    state->n = point.N;
    state->limbs = point.L;
    if (negacyclic_init(point.N, point.W, point.L, point.q.data.data(), nullptr, &state->plan) != NEGACYCLIC_OK) {
        delete state;
        raise("fherma_init");
    }
    // the harness passes pageable std::vectors: page-locked staging is made here, not in the timed run
    if (negacyclic_prepare_host(state->plan) != NEGACYCLIC_OK) {
        negacyclic_free(state->plan);
        delete state;
        raise("fherma_init");
    }
    return state;
}

fherma::Outputs fherma_run(void* opaque, const fherma::Inputs& in) {
    auto* state = static_cast<State*>(opaque);
    const size_t count = size_t(state->n) * state->limbs;
    if (in.a.data.size() != count || in.b.data.size() != count) throw std::runtime_error("wrong input size");
    // the output vector is built on the helper thread while the operands are packed and the
    // device computes; its chunks are copied in as they land
    state->output.start(count);
    const int begun = negacyclic_run_begin(state->plan, in.a.data.data(), in.b.data.data());
    fherma::Outputs out;
    out.c.shape = {int64_t(state->n), int64_t(state->limbs)};
    out.c.data = state->output.take();
    if (begun != NEGACYCLIC_OK) {
        state->output.release();
        raise("fherma_run");
    }
    const int finished = negacyclic_run_finish(state->plan, out.c.data.data());
    state->output.release();
    if (finished != NEGACYCLIC_OK) raise("fherma_run");
    return out;
}

void fherma_free(void* opaque) {
    auto* state = static_cast<State*>(opaque);
    if (!state) return;
    negacyclic_free(state->plan);
    delete state;
}
