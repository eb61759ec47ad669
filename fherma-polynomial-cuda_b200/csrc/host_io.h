// Host side of the streamed path: a persistent team of copy threads.
//
// Pageable host arrays cannot be read by the GPU's copy engines directly; the driver would
// stage them through its own pinned buffers one piece at a time (11-21 GB/s measured on a
// B200 host, against 55 GB/s from page-locked memory). The host path instead copies each
// chunk into the plan's page-locked staging buffer with several threads at once (memory
// bandwidth, not one core, is the limit: 55-80 GB/s with 8-12 threads), and the copy engine
// moves each chunk as soon as the team has packed it. The reference solves the same problem
// with persistent worker teams and AVX-512 stream copies
// (candidates/ordered-streaming/streaming_team.h:11-60); here plain memcpy slices on a
// std::thread team suffice.
//
// The team runs jobs in the order they are posted. Every worker takes part in every job (a
// job is a function of the worker index), so a job splits its work into one slice per worker.
// A job can publish finer-grained progress itself (per-chunk counters), which is how the
// launcher thread learns that chunk k is packed while later chunks are still being copied.
// Waits spin for a fixed time (kSpinTime) before they block, and the team keeps spinning between
// the jobs of one product: on the 16-vCPU host of a B200 box, once the copy threads slept, the
// device's reads of host memory slowed down several-fold (the last 3.6 MB input chunk of a
// product took 700-900 us to copy instead of 75; spinning threads keep the host's memory path
// awake), and waking a sleeping thread goes through the kernel and the hypervisor. The default
// spin (100 ms) also spans the platform harness's file I/O between two calls: behind that
// harness, fherma_run took 0.523 ms against 0.535 at N=32768/L=28, and 1.49 against 1.54 at
// N=65536/L=55, with 100 ms instead of 2 ms (4 alternating runs of 20 cases each).
#pragma once

#include <algorithm>
#include <cstdint>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#if defined(__x86_64__) || defined(__i386__)
#include <immintrin.h>
#define NEGACYCLIC_PAUSE() _mm_pause()
#else
#define NEGACYCLIC_PAUSE() std::this_thread::yield()
#endif

namespace negacyclic {

#if defined(__x86_64__) && defined(__GNUC__)
// dst[0..bytes) = src[0..bytes), writing every whole 64-byte line of the destination with a
// streaming (non-temporal) store and the partial lines at either end with memcpy. Streaming stores
// bypass the caches, so filling the page-locked staging neither evicts the caller's data nor reads
// the destination first. They are weakly ordered: the caller fences (store_fence) before it
// publishes the copy to another thread.
__attribute__((target("avx512f"))) inline void stream_copy_avx512(void* dst, const void* src, size_t bytes) {
    char* const out = static_cast<char*>(dst);
    const char* const in = static_cast<const char*>(src);
    const uintptr_t start = reinterpret_cast<uintptr_t>(out), stop = start + bytes;
    const uintptr_t lines_from = (start + 63) & ~uintptr_t(63), lines_to = stop & ~uintptr_t(63);
    if (lines_to <= lines_from) {  // no whole line inside the destination
        std::memcpy(out, in, bytes);
        return;
    }
    const size_t lead = lines_from - start, lines = (lines_to - lines_from) / 64;
    std::memcpy(out, in, lead);
    __m512i* line = reinterpret_cast<__m512i*>(out + lead);
    const char* from = in + lead;
    size_t k = 0;
    for (; k + 2 <= lines; k += 2, from += 128) {  // two lines per step
        const __m512i first = _mm512_loadu_si512(from), second = _mm512_loadu_si512(from + 64);
        _mm512_stream_si512(line + k, first);
        _mm512_stream_si512(line + k + 1, second);
    }
    if (k < lines) {
        _mm512_stream_si512(line + k, _mm512_loadu_si512(from));
        from += 64;
    }
    std::memcpy(out + (lines_to - start), from, stop - lines_to);
}
#endif

// Copy into page-locked staging: streaming stores where the CPU has AVX-512, memcpy elsewhere.
inline void stage_copy(void* dst, const void* src, size_t bytes) {
#if defined(__x86_64__) && defined(__GNUC__)
    static const bool avx512 = (__builtin_cpu_init(), __builtin_cpu_supports("avx512f"));
    if (avx512) {
        stream_copy_avx512(dst, src, bytes);
        return;
    }
#endif
    std::memcpy(dst, src, bytes);
}

// Orders this thread's earlier streaming stores before its later stores (a release publication).
inline void store_fence() {
#if defined(__x86_64__) || defined(__i386__)
    _mm_sfence();
#endif
}

class HostTeam {
public:
    using Job = std::function<void(unsigned worker, unsigned workers)>;

    // spin: how long a wait spins before it blocks (see kSpinTime)
    explicit HostTeam(unsigned workers, std::chrono::microseconds spin = kSpinTime)
        : workers_(std::max(1u, workers)), spin_(spin) {
        for (unsigned i = 0; i < workers_; ++i) threads_.emplace_back([this, i] { loop(i); });
    }

    ~HostTeam() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
            stopping_.store(true, std::memory_order_release);  // ends spinning waits at once
        }
        wake_.notify_all();
        for (auto& t : threads_) t.join();
    }

    HostTeam(const HostTeam&) = delete;
    HostTeam& operator=(const HostTeam&) = delete;

    unsigned workers() const { return workers_; }

    // Queues `job` for every worker; returns its ticket at once.
    uint64_t post(Job job) {
        uint64_t ticket;
        {
            std::lock_guard<std::mutex> lock(mu_);
            jobs_.push_back(std::move(job));
            ticket = posted_.fetch_add(1, std::memory_order_release) + 1;
        }
        wake_.notify_all();
        return ticket;
    }

    // Returns once every worker has finished job `ticket` (and, jobs running in order, every
    // job posted before it).
    void wait(uint64_t ticket) {
        const auto until = std::chrono::steady_clock::now() + spin_;
        for (uint32_t spins = 0; finished_.load(std::memory_order_acquire) < ticket; ++spins) {
            if ((spins & 63u) != 63u || std::chrono::steady_clock::now() < until) {
                NEGACYCLIC_PAUSE();
            } else {
                std::unique_lock<std::mutex> lock(mu_);
                done_.wait(lock, [&] { return finished_.load(std::memory_order_acquire) >= ticket; });
            }
        }
    }

    static constexpr std::chrono::microseconds kSpinTime{100000};  // default spinning before a wait blocks
    std::chrono::microseconds spin_time() const { return spin_; }

    // Whether job `ticket` has finished (no waiting).
    bool finished(uint64_t ticket) const { return finished_.load(std::memory_order_acquire) >= ticket; }

    // dst[0..bytes) = src[0..bytes), split over the workers; blocking.
    void copy(void* dst, const void* src, size_t bytes) {
        wait(post([=](unsigned w, unsigned n) {
            const size_t b = slice_begin(bytes, w, n), e = slice_begin(bytes, w + 1, n);
            if (e > b) std::memcpy(static_cast<char*>(dst) + b, static_cast<const char*>(src) + b, e - b);
        }));
    }

    // Writes zeros over [ptr, ptr + bytes), split over the workers: the first touch of freshly
    // mapped pages (page faults and the kernel's own zeroing) runs on every worker at once.
    void touch(void* ptr, size_t bytes) {
        wait(post([=](unsigned w, unsigned n) {
            const size_t b = slice_begin(bytes, w, n), e = slice_begin(bytes, w + 1, n);
            if (e > b) std::memset(static_cast<char*>(ptr) + b, 0, e - b);
        }));
    }

    // Start of slice w of n over `total` units, in 64-unit steps (cache lines for bytes).
    static size_t slice_begin(size_t total, unsigned w, unsigned n) {
        if (w >= n) return total;
        const size_t step = (total / n + 63) / 64 * 64;
        return std::min(total, step * w);
    }

private:
    void loop(unsigned index) {
        uint64_t next = 1;  // ticket of the next job this worker runs
        for (;;) {
            Job job;
            const auto until = std::chrono::steady_clock::now() + spin_;
            for (uint32_t spins = 0;; ++spins) {
                if (posted_.load(std::memory_order_acquire) >= next) {
                    std::lock_guard<std::mutex> lock(mu_);
                    job = jobs_[next - 1 - retired_];
                    break;
                }
                // stopping and nothing left (the acquire makes every earlier post visible)
                if (stopping_.load(std::memory_order_acquire) && posted_.load(std::memory_order_acquire) < next)
                    return;
                if ((spins & 63u) != 63u || std::chrono::steady_clock::now() < until) {
                    NEGACYCLIC_PAUSE();
                    continue;
                }
                std::unique_lock<std::mutex> lock(mu_);
                wake_.wait(lock, [&] { return stop_ || posted_.load(std::memory_order_acquire) >= next; });
                if (stop_ && posted_.load(std::memory_order_acquire) < next) return;
            }
            job(index, workers_);
            std::lock_guard<std::mutex> lock(mu_);
            if (++count_[next] == workers_) {  // last worker out retires the job
                count_.erase(next);
                finished_.store(next, std::memory_order_release);
                while (retired_ < next) {
                    jobs_.pop_front();
                    ++retired_;
                }
                done_.notify_all();
            }
            ++next;
        }
    }

    const unsigned workers_;
    const std::chrono::microseconds spin_;
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable wake_, done_;
    std::deque<Job> jobs_;             // jobs retired_+1 .. posted_
    uint64_t retired_ = 0;
    std::atomic<uint64_t> posted_{0}, finished_{0};
    std::map<uint64_t, unsigned> count_;  // workers done, per job still running
    bool stop_ = false;
    std::atomic<bool> stopping_{false};
};

// Spins until `flag` reaches `value` (acquire): one thread's short waits (the launcher waiting
// for the team to pack a chunk); yields its core after `spin`.
inline void spin_until(const std::atomic<uint32_t>& flag, uint32_t value,
                       std::chrono::microseconds spin = HostTeam::kSpinTime) {
    const auto until = std::chrono::steady_clock::now() + spin;
    for (uint32_t spins = 0; flag.load(std::memory_order_acquire) < value; ++spins) {
        if ((spins & 63u) != 63u || std::chrono::steady_clock::now() < until)
            NEGACYCLIC_PAUSE();
        else
            std::this_thread::yield();
    }
}

}  // namespace negacyclic
