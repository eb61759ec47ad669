// Host side of the streamed path: a persistent team of copy threads.
//
// Pageable host arrays cannot be read by the GPU's copy engines directly; the
// driver would stage them through its own pinned buffers one piece at a time.
// The host path instead copies each chunk into the plan's page-locked staging
// buffer with several threads at once (memory bandwidth, not one core, is the
// limit), then lets the copy engine move it while the team copies the next
// chunk. The reference solves the same problem with persistent worker teams and
// AVX-512 stream copies (candidates/ordered-streaming/streaming_team.h:11-60);
// here a plain memcpy per slice on a small std::thread pool suffices.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace negacyclic {

class CopyTeam {
public:
    explicit CopyTeam(unsigned workers) {
        for (unsigned i = 0; i < workers; ++i) threads_.emplace_back([this, i] { loop(i + 1); });
    }

    ~CopyTeam() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
            ++generation_;
        }
        start_.notify_all();
        for (auto& t : threads_) t.join();
    }

    CopyTeam(const CopyTeam&) = delete;
    CopyTeam& operator=(const CopyTeam&) = delete;

    // dst[0..bytes) = src[0..bytes), split over the workers and the calling thread.
    void copy(void* dst, const void* src, size_t bytes) { run(dst, src, 0, 0, bytes, 1); }

    // `rows` rows of row_bytes each, from src (rows src_stride bytes apart) to dst (rows
    // dst_stride bytes apart), split by rows over the workers and the calling thread.
    void copy_rows(void* dst, size_t dst_stride, const void* src, size_t src_stride, size_t row_bytes,
                   size_t rows) {
        if (rows == 1) {
            copy(dst, src, row_bytes);
            return;
        }
        run(dst, src, dst_stride, src_stride, row_bytes, rows);
    }

private:
    void run(void* dst, const void* src, size_t dst_stride, size_t src_stride, size_t row_bytes, size_t rows) {
        const unsigned parts = unsigned(threads_.size()) + 1;
        if (row_bytes * rows < (size_t(1) << 20) || parts == 1) {
            for (size_t i = 0; i < rows; ++i)
                std::memcpy(static_cast<char*>(dst) + i * dst_stride, static_cast<const char*>(src) + i * src_stride,
                            row_bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> lock(mu_);
            dst_ = static_cast<char*>(dst);
            src_ = static_cast<const char*>(src);
            dst_stride_ = dst_stride;
            src_stride_ = src_stride;
            bytes_ = row_bytes;
            rows_ = rows;
            parts_ = parts;
            pending_ = parts - 1;
            ++generation_;
        }
        start_.notify_all();
        slice(0);
        std::unique_lock<std::mutex> lock(mu_);
        done_.wait(lock, [this] { return pending_ == 0; });
    }

    void slice(unsigned index) {
        if (rows_ > 1) {  // whole rows per part
            const size_t begin = rows_ * index / parts_, end = rows_ * (index + 1) / parts_;
            for (size_t i = begin; i < end; ++i) std::memcpy(dst_ + i * dst_stride_, src_ + i * src_stride_, bytes_);
            return;
        }
        const size_t step = (bytes_ / parts_ + 63) / 64 * 64;
        const size_t begin = std::min(bytes_, step * index), end = std::min(bytes_, begin + step);
        if (index + 1 == parts_) {  // the last slice takes the remainder
            std::memcpy(dst_ + begin, src_ + begin, bytes_ - begin);
            return;
        }
        if (end > begin) std::memcpy(dst_ + begin, src_ + begin, end - begin);
    }

    void loop(unsigned index) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(mu_);
                start_.wait(lock, [&] { return generation_ != seen; });
                seen = generation_;
                if (stop_) return;
            }
            slice(index);
            {
                std::lock_guard<std::mutex> lock(mu_);
                if (--pending_ == 0) done_.notify_one();
            }
        }
    }

    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable start_, done_;
    uint64_t generation_ = 0;
    bool stop_ = false;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t dst_stride_ = 0, src_stride_ = 0, bytes_ = 0, rows_ = 1;
    unsigned parts_ = 1, pending_ = 0;
};

}  // namespace negacyclic
