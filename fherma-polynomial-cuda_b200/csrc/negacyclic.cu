// C ABI of the exact negacyclic product (include/negacyclic.h).
//
// Stage sequence of one product (device-resident; reference stages in brackets):
//   pad        operands -> [2][N][Lp], split-major rows (the host path pads chunk by chunk)
//   convert    byte-sliced u8 GEMM + REDC epilogue        [tensor_product<true>, src/solve.cu:88-142]
//   forward    merged-psi NTT per (operand, prime, t)     [high_stages/middle_stages, src/solve.cu:172-242]
//   pointwise  s x s products at each evaluation point    [middle_stages, src/solve.cu:227]
//   inverse    NTT^-1 per (prime, v), finish factor       [src/solve.cu:229-241, 199-203]
//   transpose  -> coefficient-major CRT inputs            [transpose_residues, src/solve.cu:244-253]
//   crt        byte-sliced u8 GEMM -> u64 word sums       [tensor_product<false>, src/solve.cu:603]
//   reduce     carry, CRT quotient, mod q                 [reconstruct*, src/solve.cu:323-500]
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/negacyclic.h"
#include "gemm_tc.cuh"
#include "host_plan.h"
#include "kernels.cuh"
#include "plan_internal.h"

using namespace negacyclic;

namespace negacyclic::detail {

thread_local std::string g_error;

int fail(int status, const std::string& message) {
    g_error = message;
    return status;
}

void check(cudaError_t code, const char* where) {
    if (code != cudaSuccess) throw CudaError{code, where};
}

template <class T>
void device_alloc(T*& ptr, size_t count, size_t& counter) {
    if (count == 0) count = 1;
    check(cudaMalloc(reinterpret_cast<void**>(&ptr), count * sizeof(T)), "cudaMalloc");
    counter += count * sizeof(T);
}

uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

}  // namespace negacyclic::detail

using namespace negacyclic::detail;

namespace negacyclic::detail {

constexpr uint32_t kStages = 7;  // convert, forward, pointwise, inverse, transpose, crt, reduce

// conversion GEMM over the coefficients s*j + t, t in [t_first, t_first + t_count),
// j in [first_j, first_j + span), of operands [op_first, op_first + op_count)
void enqueue_convert(negacyclic_plan& s, uint32_t t_first, uint32_t t_count, uint32_t first_j, uint32_t span,
                     cudaStream_t stream, uint32_t op_first = 0, uint32_t op_count = 2) {
    const HostPlan& h = s.host;
    Epilogue convert{};
    convert.mode = kEpilogueConvert;
    convert.residues = s.residues;
    convert.primes = s.primes;
    convert.r = s.r;
    convert.n = h.n;
    convert.status = s.status;
    const RowMap rows = RowMap::split_rows(h.n, h.n_sub, h.split, first_j, span, t_first, t_count, op_first);
    const uint32_t m = op_count * t_count * span;
    if (s.convert_engine == NEGACYCLIC_GEMM_TENSOR && gemm_tensor_accepts(s.convert_gemm, rows, m))
        launch_gemm_tensor(s.convert_gemm, convert, stream, rows, m);
    else
        launch_gemm_simt(reinterpret_cast<const uint8_t*>(s.operands), uint64_t(s.padded_limbs) * 4, rows, m,
                         s.convert_weights, 4 * s.padded_r, s.k_convert, convert, stream);
}

// CRT GEMM and reduction of coefficients [first, first + count) into d_c (rows indexed from 0 = coefficient 0)
void enqueue_output(negacyclic_plan& s, uint32_t first, uint32_t count, uint32_t* d_c, cudaStream_t stream,
                    cudaEvent_t between = nullptr) {
    const HostPlan& h = s.host;
    Epilogue crt{};
    crt.mode = kEpilogueCrt;
    crt.dots = s.dots;
    crt.words = h.words;
    crt.dots_stride = s.dots_stride;
    crt.status = s.status;
    const RowMap rows = RowMap::linear(first);
    if (s.crt_engine == NEGACYCLIC_GEMM_TENSOR && gemm_tensor_accepts(s.crt_gemm, rows, count))
        launch_gemm_tensor(s.crt_gemm, crt, stream, rows, count);
    else
        launch_gemm_simt(reinterpret_cast<const uint8_t*>(s.crt_in), uint64_t(s.padded_r) * 4, rows, count,
                         s.crt_weights, s.crt_columns, s.k_crt, crt, stream);
    if (between) check(cudaEventRecord(between, stream), "cudaEventRecord");
    ReduceParams reduce{};
    reduce.dots = s.dots + size_t(first) * s.dots_stride;
    reduce.dots_stride = s.dots_stride;
    reduce.out = d_c + size_t(first) * h.limbs;
    reduce.q = s.q;
    reduce.minus_p = s.minus_p;
    reduce.n = count;
    reduce.limbs = h.limbs;
    reduce.words = h.words;
    reduce.top_shift = h.top_shift;
    reduce.mu_low = h.mu_low;
    reduce.error_flag = s.status;
    launch_reduce(reduce, stream);
}

// forward NTTs, pointwise products, inverse NTTs, transpose, all transforms
void enqueue_middle(negacyclic_plan& s, cudaStream_t stream, cudaEvent_t* marks) {
    const HostPlan& h = s.host;
    const uint32_t n = h.n;
    uint32_t stage = 0;
    auto mark = [&]() {
        if (marks) check(cudaEventRecord(marks[stage], stream), "cudaEventRecord");
        ++stage;
    };
    launch_ntt_forward(s.residues, s.primes, s.fwd, s.r, n, h.n_sub, 0, h.split, stream);
    mark();
    launch_pointwise(s.residues, s.primes, s.zeta, s.r, n, h.n_sub, h.split, stream);
    mark();
    launch_ntt_inverse(s.residues, s.primes, s.inv, s.r, n, h.n_sub, 0, h.split, stream);
    mark();
    launch_transpose(s.residues, s.crt_in, s.r, s.padded_r, n, h.split, 0, h.n_sub, stream);
    mark();
}

// Enqueues the whole product on `stream`. `operands` already holds the padded inputs.
// `marks` (optional, kStages events) are recorded after each stage.
void enqueue_product(negacyclic_plan& s, uint32_t* d_c, cudaStream_t stream, cudaEvent_t* marks = nullptr) {
    const HostPlan& h = s.host;
    enqueue_convert(s, 0, h.split, 0, h.n_sub, stream);
    if (marks) check(cudaEventRecord(marks[0], stream), "cudaEventRecord");
    enqueue_middle(s, stream, marks ? marks + 1 : nullptr);
    enqueue_output(s, 0, h.n, d_c, stream, marks ? marks[5] : nullptr);
    if (marks) check(cudaEventRecord(marks[6], stream), "cudaEventRecord");
    check(cudaGetLastError(), "product kernels");
}

// Work-space layout of one product (256-byte aligned pieces).
struct WorkLayout {
    size_t operands, residues, crt_in, dots, result, tile_counter, total;
};

WorkLayout work_layout(const negacyclic_plan& s) {
    const HostPlan& h = s.host;
    auto align = [](size_t x) { return (x + 255) / 256 * 256; };
    WorkLayout w{};
    size_t at = 0;
    w.operands = at;
    at = align(at + size_t(2) * h.n * s.padded_limbs * 4);
    w.residues = at;
    at = align(at + size_t(2) * s.r * h.n * 4);
    w.crt_in = at;
    at = align(at + size_t(h.n) * s.padded_r * 4);
    w.dots = at;
    at = align(at + size_t(h.n) * s.dots_stride * 8);
    w.result = at;
    at = align(at + size_t(h.n) * h.limbs * 4);
    w.tile_counter = at;  // the tensor-core GEMMs of this work space run one after another
    at = align(at + 4);
    w.total = at;
    return w;
}

// Points the plan at a work space and re-encodes the GEMM tensor maps for it.
// Returns an error message, or "" on success.
std::string bind_work(negacyclic_plan& s, void* arena) {
    const HostPlan& h = s.host;
    const WorkLayout w = work_layout(s);
    uint8_t* base = static_cast<uint8_t*>(arena);
    s.operands = reinterpret_cast<uint32_t*>(base + w.operands);
    s.residues = reinterpret_cast<uint32_t*>(base + w.residues);
    s.crt_in = reinterpret_cast<uint32_t*>(base + w.crt_in);
    s.dots = reinterpret_cast<uint64_t*>(base + w.dots);
    s.result = reinterpret_cast<uint32_t*>(base + w.result);
    s.convert_engine = s.crt_engine = NEGACYCLIC_GEMM_SIMT;
    if (!s.gemm_tensor_wanted) return "";
    s.convert_gemm.tile_counter = s.crt_gemm.tile_counter = reinterpret_cast<uint32_t*>(base + w.tile_counter);
    std::string why_convert, why_crt;
    if (prepare_gemm_tensor(s.convert_gemm, reinterpret_cast<const uint8_t*>(s.operands), uint64_t(s.padded_limbs) * 4,
                            RowMap::split_rows(h.n, h.n_sub, h.split, 0, h.n_sub, 0, h.split), 2 * h.n, s.convert_weights,
                            4 * s.padded_r, s.k_convert, why_convert))
        s.convert_engine = NEGACYCLIC_GEMM_TENSOR;
    if (prepare_gemm_tensor(s.crt_gemm, reinterpret_cast<const uint8_t*>(s.crt_in), uint64_t(s.padded_r) * 4,
                            RowMap::linear(0), h.n, s.crt_weights, s.crt_columns, s.k_crt, why_crt))
        s.crt_engine = NEGACYCLIC_GEMM_TENSOR;
    if (!s.gemm_pairs_allowed) s.convert_gemm.pairs = s.crt_gemm.pairs = false;
    if (s.gemm_tensor_required &&
        (s.convert_engine != NEGACYCLIC_GEMM_TENSOR || s.crt_engine != NEGACYCLIC_GEMM_TENSOR))
        return "tensor-core GEMM not available for this point: " + why_convert + (why_convert.empty() ? "" : "; ") +
               why_crt;
    return "";
}

void enqueue_device_product(negacyclic_plan& s, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                            cudaStream_t stream) {
    launch_pad_operands(d_a, d_b, s.operands, s.host.n, s.host.limbs, s.padded_limbs, s.host.split, stream);
    enqueue_product(s, d_c, stream);
}

int cuda_failure(const CudaError& e) {
    return fail(NEGACYCLIC_ECUDA, std::string(e.where) + ": " + cudaGetErrorString(e.code));
}

int status_failure(uint32_t flags, const std::string& what) {
    if (!flags) return NEGACYCLIC_OK;
    char hex[16];
    std::snprintf(hex, sizeof hex, "0x%x", flags);
    std::string message = what.empty() ? "" : what + ": ";
    if (flags & NEGACYCLIC_STATUS_GEMM_MASK)
        message += "tensor-core GEMM pipeline wait gave up";
    else if (flags & NEGACYCLIC_STATUS_REDUCE)
        message += "reduction exceeded its proven correction bound";
    else
        message += "device status word set";
    return fail(NEGACYCLIC_ECUDA, message + " (status " + hex + ")");
}


}  // namespace negacyclic::detail

extern "C" {

const char* negacyclic_last_error(void) { return g_error.c_str(); }

int negacyclic_host_plan(uint32_t n, uint32_t limbs, const uint32_t* q, uint32_t split, uint32_t max_primes,
                         uint32_t* primes_out, uint32_t* split_out, uint32_t* n_sub_out, uint32_t* primes,
                         uint32_t* finish, uint32_t* crt_mod_q, uint32_t* minus_p_mod_q) {
    HostPlan plan;
    std::string error;
    int status = 0;
    if (!build_host_plan(n, limbs, q, split, plan, error, status)) return fail(status, error);
    const uint32_t r = uint32_t(plan.primes.size());
    if (primes_out) *primes_out = r;
    if (split_out) *split_out = plan.split;
    if (n_sub_out) *n_sub_out = plan.n_sub;
    if (max_primes == 0) return NEGACYCLIC_OK;
    if (max_primes < r) return fail(NEGACYCLIC_EINVAL, "max_primes smaller than the number of primes");
    for (uint32_t k = 0; k < r; ++k) {
        if (primes) primes[k] = plan.primes[k].p;
        if (finish) finish[k] = plan.primes[k].finish;
        if (crt_mod_q)
            std::memcpy(crt_mod_q + size_t(k) * limbs, &plan.crt_weights[size_t(k) * plan.words],
                        limbs * sizeof(uint32_t));
    }
    if (minus_p_mod_q) std::memcpy(minus_p_mod_q, plan.minus_p_mod_q.data(), limbs * sizeof(uint32_t));
    return NEGACYCLIC_OK;
}

int negacyclic_init(uint32_t n, uint32_t w, uint32_t limbs, const uint32_t* q, const negacyclic_options* opts,
                    negacyclic_plan** out) {
    if (!out) return fail(NEGACYCLIC_EINVAL, "plan output pointer is NULL");
    *out = nullptr;
    if (limbs != (w + 31) / 32)
        return fail(NEGACYCLIC_EINVAL, "invalid point: L must equal (W + 31) / 32");
    negacyclic_options o{};
    o.device = -1;
    if (opts) o = *opts;
    int device = o.device;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(NEGACYCLIC_ENODEV, "no CUDA device");
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return fail(NEGACYCLIC_ENODEV, "cannot query CUDA device " + std::to_string(device));
    if (prop.major != 10 || prop.minor != 0)
        return fail(NEGACYCLIC_ENODEV, std::string("device is not sm_100 (B200): ") + prop.name);

    auto plan = std::make_unique<negacyclic_plan>();
    plan->device = device;
    std::string error;
    int status = 0;
    if (!build_host_plan(n, limbs, q, o.split, plan->host, error, status)) return fail(status, error);
    DeviceGuard guard(device);
    negacyclic_plan& s = *plan;
    const HostPlan& h = s.host;
    s.r = uint32_t(h.primes.size());
    s.padded_r = round_up(s.r, 32);
    s.padded_limbs = round_up(limbs, 32);  // 128-byte operand rows: each TMA row read is whole L2 lines
    s.k_convert = 4 * s.padded_limbs;
    s.k_crt = 4 * s.padded_r;
    s.crt_columns = round_up(4 * h.words, 64);
    s.dots_stride = round_up(h.words, 8);
    try {
        check(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaStreamCreateWithFlags(&s.copy_in, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaStreamCreateWithFlags(&s.copy_out, cudaStreamNonBlocking), "cudaStreamCreate");
        s.chunks = host_chunks(h.n, h.n_sub, h.split);  // csrc/host_chunks.h
        for (uint32_t c = 0; c < (s.chunks > 1 ? negacyclic_plan::kMaxChunks : 1u); ++c) {
            check(cudaEventCreateWithFlags(&s.in_ready[c], cudaEventDisableTiming), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&s.out_ready[c], cudaEventDisableTiming), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&s.copied_out[c], cudaEventDisableTiming), "cudaEventCreate");
        }
        size_t tables = 0, work = 0;
        device_alloc(s.primes, s.r, tables);
        device_alloc(s.fwd, size_t(s.r) * h.n_sub, tables);
        device_alloc(s.inv, size_t(s.r) * h.n_sub, tables);
        device_alloc(s.zeta, size_t(s.r) * h.n_sub, tables);
        device_alloc(s.convert_weights, size_t(4) * s.padded_r * s.k_convert, tables);
        device_alloc(s.crt_weights, size_t(s.crt_columns) * s.k_crt, tables);
        device_alloc(s.q, limbs, tables);
        device_alloc(s.minus_p, limbs, tables);
        device_alloc(s.own_status, 64, tables);
        s.status = s.own_status;
        device_alloc(s.crt_words, size_t(s.r) * h.words, work);  // freed once the CRT weights are built
        work = 0;
        s.work_bytes = work_layout(s).total;
        if (!o.external_work) {
            check(cudaMalloc(&s.work_arena, s.work_bytes), "cudaMalloc");
            work = s.work_bytes;
        }
        s.table_bytes = tables;
        s.device_bytes = tables + work;

        std::vector<DevicePrime> primes(s.r);
        for (uint32_t k = 0; k < s.r; ++k) {
            const PrimeInfo& p = h.primes[k];
            primes[k] = DevicePrime{p.p, p.pinv, p.finish, p.finish_q, p.psi, p.r2};
        }
        cudaStream_t st = s.stream;
        check(cudaMemcpyAsync(s.primes, primes.data(), s.r * sizeof(DevicePrime), cudaMemcpyHostToDevice, st), "upload");
        check(cudaMemcpyAsync(s.q, h.q.data(), limbs * 4, cudaMemcpyHostToDevice, st), "upload q");
        check(cudaMemcpyAsync(s.minus_p, h.minus_p_mod_q.data(), limbs * 4, cudaMemcpyHostToDevice, st), "upload");
        check(cudaMemsetAsync(s.own_status, 0, 64 * sizeof(uint32_t), st), "memset");
        check(cudaMemcpyAsync(s.crt_words, h.crt_weights.data(), h.crt_weights.size() * 4, cudaMemcpyHostToDevice, st),
              "upload crt");
        launch_twiddles(s.primes, s.r, h.n_sub, s.fwd, s.inv, s.zeta, st);
        launch_convert_weights(s.primes, s.r, s.padded_r, limbs, s.k_convert, s.convert_weights, st);
        launch_crt_weights(s.crt_words, s.r, s.padded_r, h.words, s.crt_columns, s.crt_weights, st);
        check(cudaGetLastError(), "table kernels");
        check(cudaStreamSynchronize(st), "plan tables");
        cudaFree(s.crt_words);
        s.crt_words = nullptr;

        s.gemm_tensor_wanted = o.gemm != NEGACYCLIC_GEMM_SIMT;
        s.gemm_tensor_required = o.gemm == NEGACYCLIC_GEMM_TENSOR || o.gemm == NEGACYCLIC_GEMM_TENSOR_SINGLE;
        s.gemm_pairs_allowed = o.gemm != NEGACYCLIC_GEMM_TENSOR_SINGLE;
        if (s.work_arena) {
            // padding columns of the operands never reach the product (their conversion weights
            // are zero), so the arena needs no clearing; zero it anyway for deterministic dumps
            check(cudaMemsetAsync(s.work_arena, 0, s.work_bytes, st), "memset");
            check(cudaStreamSynchronize(st), "memset");
            const std::string why = bind_work(s, s.work_arena);
            if (!why.empty()) return fail(NEGACYCLIC_EINVAL, why);
        } else if (s.gemm_tensor_required) {
            // check now that the shape takes tensor cores; the real binding comes later
            void* probe = nullptr;
            check(cudaMalloc(&probe, 256), "cudaMalloc");
            const std::string why = bind_work(s, probe);
            cudaFree(probe);
            s.operands = s.residues = s.crt_in = s.result = nullptr;
            s.dots = nullptr;
            if (!why.empty()) return fail(NEGACYCLIC_EINVAL, why);
        }
    } catch (const CudaError& e) {
        cudaGetLastError();
        return e.code == cudaErrorMemoryAllocation ? fail(NEGACYCLIC_ENOMEM, "device allocation failed")
                                                   : cuda_failure(e);
    }
    *out = plan.release();
    return NEGACYCLIC_OK;
}

size_t negacyclic_work_bytes(const negacyclic_plan* s) { return s ? s->work_bytes : 0; }

int negacyclic_pipeline_status(uint32_t* flags) {
    if (!flags) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    *flags = 0;
    uint32_t* word = tensor_gemm_error_flag();
    if (!word) return fail(NEGACYCLIC_ECUDA, "cannot read the pipeline status word");
    if (cudaMemcpy(flags, word, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(word, 0, 4) != cudaSuccess)
        return fail(NEGACYCLIC_ECUDA, cudaGetErrorString(cudaGetLastError()));
    return NEGACYCLIC_OK;
}

int negacyclic_plan_status(negacyclic_plan* s, uint32_t* flags) {
    if (!s || !flags) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    *flags = 0;
    DeviceGuard guard(s->device);
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(flags, s->status, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(s->status, 0, 4) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        return fail(NEGACYCLIC_ECUDA, cudaGetErrorString(cudaGetLastError()));
    return NEGACYCLIC_OK;
}

int negacyclic_bind_work(negacyclic_plan* s, void* d_work, size_t bytes) {
    if (!s || !d_work) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (s->work_arena) return fail(NEGACYCLIC_EINVAL, "plan owns its work space");
    if (bytes < s->work_bytes) return fail(NEGACYCLIC_ESIZE, "work space smaller than negacyclic_work_bytes()");
    if (reinterpret_cast<uintptr_t>(d_work) % 256) return fail(NEGACYCLIC_EINVAL, "work space must be 256-byte aligned");
    DeviceGuard guard(s->device);
    const std::string why = bind_work(*s, d_work);
    if (!why.empty()) return fail(NEGACYCLIC_EINVAL, why);
    return NEGACYCLIC_OK;
}

int negacyclic_get_info(const negacyclic_plan* s, negacyclic_info* info) {
    if (!s || !info) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    const HostPlan& h = s->host;
    *info = negacyclic_info{};
    info->n = h.n;
    info->w = h.limbs * 32;
    info->limbs = h.limbs;
    info->primes = s->r;
    info->padded_primes = s->padded_r;
    info->split = h.split;
    info->n_sub = h.n_sub;
    info->words = h.words;
    info->gemm = (s->convert_engine == NEGACYCLIC_GEMM_TENSOR ? 1u : 0u) | (s->crt_engine == NEGACYCLIC_GEMM_TENSOR ? 2u : 0u);
    info->q_bits = h.q_bits;
    info->device_bytes = s->device_bytes;
    info->table_bytes = s->table_bytes;
    info->kernels_per_product = kStages + 1;  // + the pad kernel of the device entry point
    return NEGACYCLIC_OK;
}

int negacyclic_run_device(negacyclic_plan* s, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                          void* stream_ptr) {
    if (!s || !d_a || !d_b || !d_c) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (!s->operands) return fail(NEGACYCLIC_EINVAL, "no work space bound (negacyclic_bind_work)");
    DeviceGuard guard(s->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    try {
        enqueue_device_product(*s, d_a, d_b, d_c, stream);
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

int negacyclic_run_device_timed(negacyclic_plan* s, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                                void* stream_ptr, float* stage_ms) {
    if (!s || !d_a || !d_b || !d_c || !stage_ms) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (!s->operands) return fail(NEGACYCLIC_EINVAL, "no work space bound (negacyclic_bind_work)");
    DeviceGuard guard(s->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    cudaEvent_t events[kStages + 2] = {};
    int status = NEGACYCLIC_OK;
    try {
        for (auto& e : events) check(cudaEventCreate(&e), "cudaEventCreate");
        check(cudaEventRecord(events[0], stream), "cudaEventRecord");
        launch_pad_operands(d_a, d_b, s->operands, s->host.n, s->host.limbs, s->padded_limbs, s->host.split,
                            stream);
        check(cudaEventRecord(events[1], stream), "cudaEventRecord");
        enqueue_product(*s, d_c, stream, events + 2);
        check(cudaEventSynchronize(events[kStages + 1]), "product");
        for (uint32_t i = 0; i <= kStages; ++i)
            check(cudaEventElapsedTime(&stage_ms[i], events[i], events[i + 1]), "cudaEventElapsedTime");
    } catch (const CudaError& e) {
        status = cuda_failure(e);
    }
    for (auto& e : events)
        if (e) cudaEventDestroy(e);
    return status;
}

}  // extern "C"

namespace negacyclic::detail {

bool page_locked(const void* ptr) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost || attr.type == cudaMemoryTypeManaged;
}

// Page-locked staging and the copy team of the host path, made on first use.
// NEGACYCLIC_HOST_THREADS sets the team's size (by default up to 6 of the host's cores), and
// NEGACYCLIC_HOST_SPIN_US how long its threads spin before they sleep (default 100000 us).
// Host memory bandwidth, shared with the copy engines and the caller's output fill, is the limit:
// on a 16-core B200 host, fherma_run at N=65536, L=55 took 1.40-1.46 ms with 6 threads against
// 1.52-1.62 with 8, 1.60-1.67 with 4 and 1.91 with 3 (0.65-0.77 ms at N=32768, L=28).
void ensure_staging(negacyclic_plan& s) {
    const size_t words = size_t(s.host.n) * s.host.limbs;
    if (!s.stage_in) check(cudaHostAlloc(&s.stage_in, 2 * words * 4, cudaHostAllocWriteCombined), "cudaHostAlloc");
    if (!s.stage_out) check(cudaHostAlloc(&s.stage_out, words * 4, cudaHostAllocDefault), "cudaHostAlloc");
    if (!s.team) {
        const unsigned hw = std::max(3u, std::thread::hardware_concurrency());
        unsigned workers = std::min(6u, hw - 2);
        if (const char* env = getenv("NEGACYCLIC_HOST_THREADS"))
            workers = std::max(1u, std::min(64u, unsigned(std::strtoul(env, nullptr, 10))));
        std::chrono::microseconds spin = HostTeam::kSpinTime;
        if (const char* env = getenv("NEGACYCLIC_HOST_SPIN_US"))
            spin = std::chrono::microseconds(std::min<unsigned long>(10000000ul, std::strtoul(env, nullptr, 10)));
        s.team = std::make_unique<HostTeam>(workers, spin);
    }
}

// The plan's shape for the chunk lists (csrc/host_chunks.h).
ChunkShape chunk_shape(const negacyclic_plan& s) {
    return ChunkShape{s.host.n, s.host.n_sub, s.host.split, s.host.limbs, s.chunks};
}

void copy_rows_async(void* dst, size_t dpitch, const void* src, size_t spitch, size_t row, uint32_t rows,
                     cudaMemcpyKind kind, cudaStream_t stream, const char* what) {
    if (dpitch == row && spitch == row)
        check(cudaMemcpyAsync(dst, src, row * rows, kind, stream), what);
    else
        check(cudaMemcpy2DAsync(dst, dpitch, src, spitch, row, rows, kind, stream), what);
}

// Enqueues a host product. Inputs: page-locked arrays go straight to the copy engine,
// pageable ones through stage_in (the team copies chunk k+1 while chunk k is in flight).
// Output: straight into c when c is page-locked, else into stage_out for host_finish.
void host_begin(negacyclic_plan& s, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    const HostPlan& h = s.host;
    const size_t row = size_t(h.limbs) * 4, words = size_t(h.n) * h.limbs;
    const uint32_t split = h.split, n_sub = h.n_sub;
    cudaStream_t st = s.stream;
    const bool a_locked = page_locked(a), b_locked = page_locked(b);
    s.outputs_staged = !(c && page_locked(c));
    if (!a_locked || !b_locked || s.outputs_staged) ensure_staging(s);
    if (s.pack_ticket) {  // a previous call that failed part-way may still be packing
        s.team->wait(s.pack_ticket);
        s.pack_ticket = 0;
    }
    if (!s.status_host) check(cudaHostAlloc(&s.status_host, 64, cudaHostAllocDefault), "cudaHostAlloc");
    *static_cast<volatile uint32_t*>(s.status_host) = 0;  // the previous call's stream has finished
    check(cudaMemsetAsync(s.status, 0, 4, st), "memset");
    const uint32_t* src[2] = {a, b};
    const bool locked[2] = {a_locked, b_locked};
    // rows land unpadded (straight in the operands when they need neither padding nor
    // permutation) and are padded on the device; the CRT word-sum buffer, written only after
    // every chunk is converted, stages them
    std::vector<InChunk> in;
    std::vector<OutChunk> out;
    const bool ordered = transform_ordered_input(chunk_shape(s));
    stream_chunks(chunk_shape(s), ordered, in, out);
    uint32_t pieces[negacyclic_plan::kMaxChunks] = {};  // pack pieces per input chunk
    if (!a_locked || !b_locked) {
        // One pack job over pieces of about kPieceBytes of the pageable operands, claimed in chunk
        // order from a shared counter (a descheduled worker holds up at most the piece it has).
        // Contiguous ranges (narrow rows) are copied with streaming stores: behind the reference's
        // harness, fherma_run took 0.465 against 0.517 ms at N=32768/L=28 and 1.330 against 1.396
        // ms at N=65536/L=55 (4 alternating runs of 20 cases). The row gather of wide rows keeps
        // memcpy: with streaming stores fherma_run at N=65536/L=1747 took 80-90 ms against 77.
        // packed[k] counts chunk k's pieces done, and the loops below hand chunk k to the copy
        // engine as soon as all of them are, while later chunks are still being packed.
        constexpr size_t kPieceBytes = 256 << 10;
        const uint32_t per_piece = uint32_t(std::max<size_t>(1, kPieceBytes / row));  // rows per piece
        const uint32_t operands = (a_locked ? 0u : 1u) + (b_locked ? 0u : 1u);
        std::vector<uint32_t> first_piece(in.size() + 1, 0);
        for (uint32_t k = 0; k < in.size(); ++k) {  // pageable operands of chunk k x its pieces each
            const uint32_t ops = in[k].op == InChunk::kBothOperands ? operands : (locked[in[k].op] ? 0u : 1u);
            pieces[k] = ops * ((in[k].span + per_piece - 1) / per_piece);
            first_piece[k + 1] = first_piece[k] + pieces[k];
            s.packed[k].store(0, std::memory_order_relaxed);
        }
        s.next_piece.store(0, std::memory_order_relaxed);
        uint32_t* stage = s.stage_in;
        const uint32_t n = h.n, limbs = h.limbs, total = first_piece.back();
        std::atomic<uint32_t>* packed = s.packed;
        std::atomic<uint32_t>* next = &s.next_piece;
        s.pack_ticket = s.team->post([=](unsigned, unsigned) {
            uint32_t k = 0;
            for (uint32_t piece = next->fetch_add(1, std::memory_order_relaxed); piece < total;
                 piece = next->fetch_add(1, std::memory_order_relaxed)) {
                while (piece >= first_piece[k + 1]) ++k;
                const InChunk ch = in[k];
                const uint32_t local = piece - first_piece[k], per_op = (ch.span + per_piece - 1) / per_piece;
                const int op = ch.op != InChunk::kBothOperands ? int(ch.op)
                               : operands == 2                 ? int(local / per_op)
                                                               : (a_locked ? 1 : 0);
                const size_t first = size_t(local % per_op) * per_piece;
                const size_t last = std::min<size_t>(ch.span, first + per_piece);
                if (ordered) {  // gather rows s*j + t to their split-major places t*N' + j
                    const size_t host_row0 = size_t(split) * ch.j0 + ch.t, buf_row0 = size_t(ch.t) * n_sub + ch.j0;
                    const uint32_t* from = src[op] + host_row0 * limbs;
                    uint32_t* to = stage + (op * size_t(n) + buf_row0) * limbs;
                    for (size_t j = first; j < last; ++j) std::memcpy(to + j * limbs, from + j * split * limbs, row);
                } else {  // a contiguous coefficient range, with streaming stores
                    const size_t at = (size_t(ch.j0) + first) * limbs;
                    stage_copy(stage + op * size_t(n) * limbs + at, src[op] + at, (last - first) * row);
                }
                store_fence();  // the streaming stores land before the piece is counted
                packed[k].fetch_add(1, std::memory_order_release);
            }
        });
    }
    if (ordered) {
        const bool direct = s.padded_limbs == h.limbs;
        uint32_t* staged = direct ? s.operands : reinterpret_cast<uint32_t*>(s.dots);
        for (uint32_t k = 0; k < in.size(); ++k) {
            const InChunk ch = in[k];
            const size_t host_row0 = size_t(split) * ch.j0 + ch.t, buf_row0 = size_t(ch.t) * n_sub + ch.j0;
            spin_until(s.packed[k], pieces[k], s.team ? s.team->spin_time() : HostTeam::kSpinTime);
            for (int op = 0; op < 2; ++op) {
                const uint32_t* from = src[op] + host_row0 * h.limbs;
                size_t pitch = split * row;
                if (!locked[op]) {  // packed into stage_in at the rows' split-major places
                    from = s.stage_in + (op * size_t(h.n) + buf_row0) * h.limbs;
                    pitch = row;
                }
                copy_rows_async(staged + (op * size_t(h.n) + buf_row0) * h.limbs, row, from, pitch, row, ch.span,
                                cudaMemcpyHostToDevice, s.copy_in, "copy in");
            }
            check(cudaEventRecord(s.in_ready[k], s.copy_in), "cudaEventRecord");
            check(cudaStreamWaitEvent(st, s.in_ready[k], 0), "cudaStreamWaitEvent");
            if (!direct)
                launch_pad_rows(staged, s.operands, h.n, h.limbs, s.padded_limbs, 1, uint32_t(buf_row0), ch.span, st);
            enqueue_convert(s, ch.t, 1, ch.j0, ch.span, st);
            if (k + 1 == in.size() || in[k + 1].t != ch.t)  // transform t complete: its forward NTTs
                launch_ntt_forward(s.residues, s.primes, s.fwd, s.r, h.n, n_sub, ch.t, 1, st);
        }
    } else {
        const bool direct = s.padded_limbs == h.limbs && split == 1;
        uint32_t* staged = direct ? s.operands : reinterpret_cast<uint32_t*>(s.dots);
        for (uint32_t k = 0; k < in.size(); ++k) {
            const size_t first = in[k].j0, count = in[k].span, bytes = count * row;  // coefficient range
            const uint32_t op_first = in[k].op == InChunk::kBothOperands ? 0u : in[k].op;
            const uint32_t op_count = in[k].op == InChunk::kBothOperands ? 2u : 1u;
            spin_until(s.packed[k], pieces[k], s.team ? s.team->spin_time() : HostTeam::kSpinTime);
            for (uint32_t op = op_first; op < op_first + op_count; ++op) {
                const uint32_t* from = src[op] + first * h.limbs;
                if (!locked[op]) from = s.stage_in + op * words + first * h.limbs;  // packed by the team
                check(cudaMemcpyAsync(staged + op * words + first * h.limbs, from, bytes, cudaMemcpyHostToDevice,
                                      s.copy_in),
                      "copy in");
            }
            check(cudaEventRecord(s.in_ready[k], s.copy_in), "cudaEventRecord");
            check(cudaStreamWaitEvent(st, s.in_ready[k], 0), "cudaStreamWaitEvent");
            if (!direct)
                launch_pad_rows(staged, s.operands, h.n, h.limbs, s.padded_limbs, split, uint32_t(first),
                                uint32_t(count), st, op_first, op_count);
            // coefficients [first, first + count): j in [first / s, (first + count) / s) of every transform
            enqueue_convert(s, 0, split, uint32_t(first / split), uint32_t(count / split), st, op_first, op_count);
            if (k + 1 == in.size() || in[k + 1].op != in[k].op)  // these operands are complete
                launch_ntt_forward(s.residues, s.primes, s.fwd, s.r, h.n, n_sub, 0, split, st, op_first, op_count);
        }
    }
    launch_pointwise(s.residues, s.primes, s.zeta, s.r, h.n, n_sub, split, st);
    launch_ntt_inverse(s.residues, s.primes, s.inv, s.r, h.n, n_sub, 0, split, st);
    // outputs: CRT GEMM and reduction per chunk, each chunk's copy-out overlapping the next
    // chunk's work. With wide rows the transpose also goes chunk by chunk, so only the first
    // chunk's share sits between the inverse NTT and the first copy-out.
    uint32_t* dst = s.outputs_staged ? s.stage_out : c;
    const bool transpose_per_chunk = wide_rows(chunk_shape(s));
    if (!transpose_per_chunk) launch_transpose(s.residues, s.crt_in, s.r, s.padded_r, h.n, split, 0, n_sub, st);
    for (uint32_t k = 0; k <= out.size(); ++k) {
        if (k < out.size()) {
            if (transpose_per_chunk)  // chunk coefficients are whole multiples of s
                launch_transpose(s.residues, s.crt_in, s.r, s.padded_r, h.n, split, out[k].first / split,
                                 out[k].count / split, st);
            enqueue_output(s, out[k].first, out[k].count, s.result, st);
            check(cudaEventRecord(s.out_ready[k], st), "cudaEventRecord");
        }
        if (k >= 1) {
            const size_t first = out[k - 1].first;
            check(cudaStreamWaitEvent(s.copy_out, s.out_ready[k - 1], 0), "cudaStreamWaitEvent");
            check(cudaMemcpyAsync(dst + first * h.limbs, s.result + first * h.limbs, size_t(out[k - 1].count) * row,
                                  cudaMemcpyDeviceToHost, s.copy_out),
                  "copy c");
            check(cudaEventRecord(s.copied_out[k - 1], s.copy_out), "cudaEventRecord");
        }
    }
    // every kernel that writes the status word runs on st: its copy follows the last of them
    check(cudaMemcpyAsync(s.status_host, s.status, 4, cudaMemcpyDeviceToHost, st), "status word");
    check(cudaGetLastError(), "product kernels");
}

// Waits for a host product; the team copies each staged output chunk into c as soon as its
// copy-out has completed.
int host_finish(negacyclic_plan& s, uint32_t* c) {
    const HostPlan& h = s.host;
    if (s.pack_ticket) {  // every chunk was issued only after it was packed: the job is done
        s.team->wait(s.pack_ticket);
        s.pack_ticket = 0;
    }
    if (s.outputs_staged) {
        std::vector<InChunk> in;
        std::vector<OutChunk> out;
        stream_chunks(chunk_shape(s), false, in, out);  // the output chunks do not depend on the input order
        // one unpack job per output chunk, posted as soon as its copy-out has completed: the
        // workers copy their slices of it into c while later chunks are still on the way (and
        // sleep, instead of spinning, while the device computes)
        const uint32_t limbs = h.limbs;
        const uint32_t* stage = s.stage_out;
        std::string failed;
        uint64_t ticket = 0;
        for (uint32_t k = 0; k < out.size(); ++k) {
            const cudaError_t e = cudaEventSynchronize(s.copied_out[k]);
            if (e != cudaSuccess) {
                failed = cudaGetErrorString(e);
                break;
            }
            const size_t words = size_t(out[k].count) * limbs, at = size_t(out[k].first) * limbs;
            ticket = s.team->post([=](unsigned w, unsigned workers) {
                const size_t b = HostTeam::slice_begin(words, w, workers), e = HostTeam::slice_begin(words, w + 1, workers);
                if (e > b) std::memcpy(c + at + b, stage + at + b, (e - b) * 4);
            });
        }
        if (ticket) s.team->wait(ticket);
        if (!failed.empty()) return fail(NEGACYCLIC_ECUDA, "copy c: " + failed);
    }
    check(cudaStreamSynchronize(s.copy_out), "product");
    check(cudaStreamSynchronize(s.stream), "product");
    const uint32_t flags = *static_cast<volatile const uint32_t*>(s.status_host);  // landed with s.stream
    return status_failure(flags);
}

}  // namespace negacyclic::detail

extern "C" {

int negacyclic_run(negacyclic_plan* s, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (!s || !a || !b || !c) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (!s->operands) return fail(NEGACYCLIC_EINVAL, "no work space bound (negacyclic_bind_work)");
    DeviceGuard guard(s->device);
    try {
        host_begin(*s, a, b, c);
        return host_finish(*s, c);
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
}

int negacyclic_prepare_host(negacyclic_plan* s) {
    if (!s) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (!s->operands) return fail(NEGACYCLIC_EINVAL, "no work space bound (negacyclic_bind_work)");
    DeviceGuard guard(s->device);
    try {
        ensure_staging(*s);
        // warm-up: 0 * 0 through the host path (page-locked inputs, staged output), which
        // loads every kernel of the path and touches the staging pages once
        const size_t words = size_t(s->host.n) * s->host.limbs;
        std::memset(s->stage_in, 0, 2 * words * 4);
        host_begin(*s, s->stage_in, s->stage_in + words, nullptr);
        check(cudaStreamSynchronize(s->copy_out), "warm-up");
        check(cudaStreamSynchronize(s->stream), "warm-up");
        uint32_t flags = 0;
        check(cudaMemcpy(&flags, s->status, 4, cudaMemcpyDeviceToHost), "warm-up");
        if (flags) return status_failure(flags, "warm-up product");
        for (size_t i = 0; i < words; i += 4096)
            if (s->stage_out[i] != 0) return fail(NEGACYCLIC_ECUDA, "warm-up product of zeros is not zero");
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

int negacyclic_run_begin(negacyclic_plan* s, const uint32_t* a, const uint32_t* b) {
    if (!s || !a || !b) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (!s->operands) return fail(NEGACYCLIC_EINVAL, "no work space bound (negacyclic_bind_work)");
    DeviceGuard guard(s->device);
    try {
        host_begin(*s, a, b, nullptr);
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

int negacyclic_run_finish(negacyclic_plan* s, uint32_t* c) {
    if (!s || !c) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    DeviceGuard guard(s->device);
    try {
        return host_finish(*s, c);
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
}

int negacyclic_host_touch(negacyclic_plan* s, void* ptr, size_t bytes) {
    if (!s || (!ptr && bytes)) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    try {
        ensure_staging(*s);
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    s->team->touch(ptr, bytes);
    return NEGACYCLIC_OK;
}

void negacyclic_free(negacyclic_plan* plan) { delete plan; }

int negacyclic_debug_read(negacyclic_plan* s, int which, void* host, size_t* bytes) {
    if (!s || !bytes) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    const HostPlan& h = s->host;
    const void* src = nullptr;
    size_t size = 0;
    switch (which) {
        case 0: src = s->residues; size = size_t(2) * s->r * h.n * 4; break;
        case 1: src = s->crt_in; size = size_t(h.n) * s->padded_r * 4; break;
        case 2: src = s->dots; size = size_t(h.n) * h.words * 8; break;
        default: return fail(NEGACYCLIC_EINVAL, "unknown buffer");
    }
    if (!host) {
        *bytes = size;
        return NEGACYCLIC_OK;
    }
    if (*bytes < size) return fail(NEGACYCLIC_EINVAL, "host buffer too small");
    DeviceGuard guard(s->device);
    cudaError_t e = which == 2  // word sums: rows of dots_stride words on the device, words returned
                        ? cudaMemcpy2D(host, size_t(h.words) * 8, src, size_t(s->dots_stride) * 8, size_t(h.words) * 8,
                                       h.n, cudaMemcpyDeviceToHost)
                        : cudaMemcpy(host, src, size, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(NEGACYCLIC_ECUDA, cudaGetErrorString(e));
    *bytes = size;
    return NEGACYCLIC_OK;
}

int negacyclic_gemm_u8(const uint8_t* d_a, const uint8_t* d_b, int32_t* d_d, uint32_t m, uint32_t n, uint32_t k,
                       uint32_t engine, void* stream_ptr) {
    if (!d_a || !d_b || !d_d || k % 16 || !m || !n || !k) return fail(NEGACYCLIC_EINVAL, "bad GEMM arguments");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    Epilogue raw{};
    raw.mode = kEpilogueRaw;
    raw.raw = d_d;
    raw.raw_ld = n;
    RowMap rows = RowMap::linear(0);
    try {
        if (engine == NEGACYCLIC_GEMM_TENSOR || engine == NEGACYCLIC_GEMM_TENSOR_SINGLE) {
            TensorGemmPlan plan;
            std::string why;
            if (!prepare_gemm_tensor(plan, d_a, k, rows, m, d_b, n, k, why))
                return fail(NEGACYCLIC_EINVAL, "tensor GEMM unavailable: " + why);
            launch_gemm_tensor(plan, raw, stream, rows, m, engine == NEGACYCLIC_GEMM_TENSOR, 0, kNoWithheldStep);
        } else {
            launch_gemm_simt(d_a, k, rows, m, d_b, n, k, raw, stream);
        }
        check(cudaGetLastError(), "gemm");
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

int negacyclic_gemm_u8_withheld(const uint8_t* d_a, const uint8_t* d_b, int32_t* d_d, uint32_t m, uint32_t n,
                                uint32_t k, uint32_t engine, uint64_t limit_cycles, uint32_t withheld_step,
                                uint32_t* flags, double* elapsed_ms) {
    if (!d_a || !d_b || !d_d || !flags || k % 16 || !m || !n || !k || !limit_cycles || limit_cycles > (1ull << 40))
        return fail(NEGACYCLIC_EINVAL, "bad GEMM arguments");
    if (engine != NEGACYCLIC_GEMM_TENSOR && engine != NEGACYCLIC_GEMM_TENSOR_SINGLE)
        return fail(NEGACYCLIC_EINVAL, "the withheld-stage check applies to the tensor-core engines");
    *flags = 0;
    uint32_t* status = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    int result = NEGACYCLIC_OK;
    try {
        TensorGemmPlan plan;
        std::string why;
        const RowMap rows = RowMap::linear(0);
        if (!prepare_gemm_tensor(plan, d_a, k, rows, m, d_b, n, k, why))
            return fail(NEGACYCLIC_EINVAL, "tensor GEMM unavailable: " + why);
        check(cudaMalloc(&status, sizeof(uint32_t)), "cudaMalloc");
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaEventCreate(&start), "cudaEventCreate");
        check(cudaEventCreate(&stop), "cudaEventCreate");
        check(cudaMemsetAsync(status, 0, sizeof(uint32_t), stream), "memset");
        Epilogue raw{};
        raw.mode = kEpilogueRaw;
        raw.raw = d_d;
        raw.raw_ld = n;
        raw.status = status;
        check(cudaEventRecord(start, stream), "cudaEventRecord");
        launch_gemm_tensor(plan, raw, stream, rows, m, engine == NEGACYCLIC_GEMM_TENSOR, (long long)limit_cycles,
                           withheld_step);
        check(cudaGetLastError(), "gemm");
        check(cudaEventRecord(stop, stream), "cudaEventRecord");
        check(cudaStreamSynchronize(stream), "gemm");
        float ms = 0;
        check(cudaEventElapsedTime(&ms, start, stop), "cudaEventElapsedTime");
        if (elapsed_ms) *elapsed_ms = ms;
        check(cudaMemcpy(flags, status, sizeof(uint32_t), cudaMemcpyDeviceToHost), "status word");
    } catch (const CudaError& e) {
        result = cuda_failure(e);
    }
    if (start) cudaEventDestroy(start);
    if (stop) cudaEventDestroy(stop);
    if (stream) cudaStreamDestroy(stream);
    if (status) cudaFree(status);
    if (result == NEGACYCLIC_OK && *flags) result = status_failure(*flags, "GEMM");
    return result;
}

}  // extern "C"
