// Internal view of a plan, shared by the C-ABI entry points, the batched form
// and the serving loop (not part of the public ABI).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/negacyclic.h"
#include "gemm_tc.cuh"
#include "host_plan.h"
#include "host_chunks.h"
#include "host_io.h"
#include "kernels.cuh"

#include <atomic>
#include <memory>

// The C ABI's opaque plan (include/negacyclic.h).
struct negacyclic_plan {
    int device = 0;
    negacyclic::HostPlan host;
    uint32_t r = 0, padded_r = 0, padded_limbs = 0, k_convert = 0, k_crt = 0, crt_columns = 0;
    uint32_t dots_stride = 0;  // words per row of the CRT word sums: L + 5 rounded up to 8
    uint32_t convert_engine = NEGACYCLIC_GEMM_SIMT, crt_engine = NEGACYCLIC_GEMM_SIMT;
    negacyclic::DevicePrime* primes = nullptr;
    uint2 *fwd = nullptr, *inv = nullptr, *zeta = nullptr;
    uint8_t *convert_weights = nullptr, *crt_weights = nullptr;
    uint32_t *q = nullptr, *minus_p = nullptr, *crt_words = nullptr;
    // per-product work space: one arena, owned or bound by the caller (batches, servers)
    uint32_t *operands = nullptr, *residues = nullptr, *crt_in = nullptr, *result = nullptr;
    uint64_t* dots = nullptr;
    // status word of this plan's products (NEGACYCLIC_STATUS_* bits): the reduce kernel and both
    // tensor GEMMs set bits in it; allocated with the tables, or pointed into a batch's array
    uint32_t* status = nullptr;
    uint32_t* own_status = nullptr;
    void* work_arena = nullptr;  // owned arena (nullptr when the work space is external)
    size_t work_bytes = 0;
    bool gemm_tensor_wanted = true, gemm_tensor_required = false, gemm_pairs_allowed = true;
    cudaStream_t stream = nullptr, copy_in = nullptr, copy_out = nullptr;
    static constexpr uint32_t kMaxChunks = negacyclic::kMaxHostChunks;
    uint32_t chunks = 1;  // coefficient chunks of the streamed host path
    cudaEvent_t in_ready[kMaxChunks] = {};
    cudaEvent_t out_ready[kMaxChunks] = {};
    cudaEvent_t copied_out[kMaxChunks] = {};
    // host path with pageable arrays: page-locked staging and a copy team (made on first use)
    uint32_t* stage_in = nullptr;   // [2][N][L], write-combined
    uint32_t* stage_out = nullptr;  // [N][L]
    // the host path's copy of the status word, written on `stream` after the last kernel, so
    // that reading it costs no extra round trip once the stream has finished
    uint32_t* status_host = nullptr;
    std::unique_ptr<negacyclic::HostTeam> team;
    std::atomic<uint32_t> packed[kMaxChunks] = {};  // pieces of input chunk k packed
    std::atomic<uint32_t> next_piece{0};            // next unclaimed piece of the running pack job
    uint64_t pack_ticket = 0;                       // the running call's pack job (0: none)
    bool outputs_staged = false;    // the running host product copies c through stage_out
    size_t device_bytes = 0, table_bytes = 0;
    negacyclic::TensorGemmPlan convert_gemm, crt_gemm;

    ~negacyclic_plan() {
        int previous = 0;
        cudaGetDevice(&previous);
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (copy_in) cudaStreamSynchronize(copy_in);
        if (copy_out) cudaStreamSynchronize(copy_out);
        void* buffers[] = {primes, fwd, inv, zeta, convert_weights, crt_weights, q, minus_p, crt_words, own_status,
                           work_arena};
        for (void* ptr : buffers)
            if (ptr) cudaFree(ptr);
        for (uint32_t c = 0; c < kMaxChunks; ++c) {
            if (in_ready[c]) cudaEventDestroy(in_ready[c]);
            if (out_ready[c]) cudaEventDestroy(out_ready[c]);
            if (copied_out[c]) cudaEventDestroy(copied_out[c]);
        }
        if (stage_in) cudaFreeHost(stage_in);
        if (stage_out) cudaFreeHost(stage_out);
        if (status_host) cudaFreeHost(status_host);
        team.reset();
        if (stream) cudaStreamDestroy(stream);
        if (copy_in) cudaStreamDestroy(copy_in);
        if (copy_out) cudaStreamDestroy(copy_out);
        cudaSetDevice(previous);
    }
};

namespace negacyclic::detail {

struct CudaError {
    cudaError_t code;
    const char* where;
};

void check(cudaError_t code, const char* where);
int fail(int status, const std::string& message);
int cuda_failure(const CudaError& e);
// NEGACYCLIC_OK for a zero status word, else NEGACYCLIC_ECUDA with a message naming what failed
// (`what` prefixes the message, e.g. the batch instance)
int status_failure(uint32_t flags, const std::string& what = "");

struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        cudaGetDevice(&previous);
        if (previous != device) cudaSetDevice(device);
    }
    ~DeviceGuard() {
        if (previous >= 0) cudaSetDevice(previous);
    }
};

// Points the plan at a work space and re-encodes its GEMM tensor maps ("" on success).
std::string bind_work(negacyclic_plan& s, void* arena);
// The device product of negacyclic_run_device: pad, convert, NTTs, CRT, reduce, on `stream`.
void enqueue_device_product(negacyclic_plan& s, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                            cudaStream_t stream);

}  // namespace negacyclic::detail
