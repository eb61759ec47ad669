// C ABI of the exact negacyclic product (include/negacyclic.h).
//
// Stage sequence of one product (device-resident; reference stages in brackets):
//   pad        operands -> [2][N][Lp] (only when L % 4 != 0; the host path pads during H2D)
//   convert    byte-sliced u8 GEMM + REDC epilogue        [tensor_product<true>, src/solve.cu:88-142]
//   forward    merged-psi NTT per (operand, prime, t)     [high_stages/middle_stages, src/solve.cu:172-242]
//   pointwise  s x s products at each evaluation point    [middle_stages, src/solve.cu:227]
//   inverse    NTT^-1 per (prime, v), finish factor       [src/solve.cu:229-241, 199-203]
//   transpose  -> coefficient-major CRT inputs            [transpose_residues, src/solve.cu:244-253]
//   crt        byte-sliced u8 GEMM -> u64 word sums       [tensor_product<false>, src/solve.cu:603]
//   reduce     carry, CRT quotient, mod q                 [reconstruct*, src/solve.cu:323-500]
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/negacyclic.h"
#include "gemm_tc.cuh"
#include "host_plan.h"
#include "kernels.cuh"

using namespace negacyclic;

namespace {

thread_local std::string g_error;

int fail(int status, const std::string& message) {
    g_error = message;
    return status;
}

struct CudaError {
    cudaError_t code;
    const char* where;
};

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

}  // namespace

struct negacyclic_plan {
    int device = 0;
    HostPlan host;
    uint32_t r = 0, padded_r = 0, padded_limbs = 0, k_convert = 0, k_crt = 0, crt_columns = 0;
    uint32_t convert_engine = NEGACYCLIC_GEMM_SIMT, crt_engine = NEGACYCLIC_GEMM_SIMT;
    DevicePrime* primes = nullptr;
    uint2 *fwd = nullptr, *inv = nullptr, *zeta = nullptr;
    uint8_t *convert_weights = nullptr, *crt_weights = nullptr;
    uint32_t *q = nullptr, *minus_p = nullptr, *crt_words = nullptr;
    uint32_t *operands = nullptr, *residues = nullptr, *crt_in = nullptr, *result = nullptr;
    uint64_t* dots = nullptr;
    uint32_t* error_flag = nullptr;
    cudaStream_t stream = nullptr, copy_in = nullptr, copy_out = nullptr;
    static constexpr uint32_t kMaxChunks = 16;
    uint32_t chunks = 1;  // coefficient chunks of the streamed host path
    cudaEvent_t in_ready[kMaxChunks] = {}, out_ready[kMaxChunks] = {};
    size_t device_bytes = 0, table_bytes = 0;
    TensorGemmPlan convert_gemm, crt_gemm;

    ~negacyclic_plan() {
        int previous = 0;
        cudaGetDevice(&previous);
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        void* buffers[] = {primes, fwd, inv, zeta, convert_weights, crt_weights, q, minus_p, crt_words,
                           operands, residues, crt_in, result, dots, error_flag};
        for (void* ptr : buffers)
            if (ptr) cudaFree(ptr);
        if (copy_in) cudaStreamSynchronize(copy_in);
        if (copy_out) cudaStreamSynchronize(copy_out);
        for (uint32_t c = 0; c < kMaxChunks; ++c) {
            if (in_ready[c]) cudaEventDestroy(in_ready[c]);
            if (out_ready[c]) cudaEventDestroy(out_ready[c]);
        }
        if (stream) cudaStreamDestroy(stream);
        if (copy_in) cudaStreamDestroy(copy_in);
        if (copy_out) cudaStreamDestroy(copy_out);
        cudaSetDevice(previous);
    }
};

namespace {

constexpr uint32_t kStages = 7;  // convert, forward, pointwise, inverse, transpose, crt, reduce

// conversion GEMM over the coefficients s*j + t, j in [first_j, first_j + span), all t, both operands
void enqueue_convert(negacyclic_plan& s, uint32_t first_j, uint32_t span, cudaStream_t stream) {
    const HostPlan& h = s.host;
    Epilogue convert{};
    convert.mode = kEpilogueConvert;
    convert.residues = s.residues;
    convert.primes = s.primes;
    convert.r = s.r;
    convert.n = h.n;
    const RowMap rows = RowMap::split_rows(h.n, h.n_sub, h.split, first_j, span);
    const uint32_t m = 2 * h.split * span;
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
    const RowMap rows = RowMap::linear(first);
    if (s.crt_engine == NEGACYCLIC_GEMM_TENSOR && gemm_tensor_accepts(s.crt_gemm, rows, count))
        launch_gemm_tensor(s.crt_gemm, crt, stream, rows, count);
    else
        launch_gemm_simt(reinterpret_cast<const uint8_t*>(s.crt_in), uint64_t(s.padded_r) * 4, rows, count,
                         s.crt_weights, s.crt_columns, s.k_crt, crt, stream);
    if (between) check(cudaEventRecord(between, stream), "cudaEventRecord");
    ReduceParams reduce{};
    reduce.dots = s.dots + size_t(first) * h.words;
    reduce.out = d_c + size_t(first) * h.limbs;
    reduce.q = s.q;
    reduce.minus_p = s.minus_p;
    reduce.n = count;
    reduce.limbs = h.limbs;
    reduce.words = h.words;
    reduce.top_shift = h.top_shift;
    reduce.mu_low = h.mu_low;
    reduce.error_flag = s.error_flag;
    launch_reduce(reduce, stream);
}

// forward NTTs, pointwise products, inverse NTTs, transpose
void enqueue_middle(negacyclic_plan& s, cudaStream_t stream, cudaEvent_t* marks) {
    const HostPlan& h = s.host;
    const uint32_t n = h.n;
    uint32_t stage = 0;
    auto mark = [&]() {
        if (marks) check(cudaEventRecord(marks[stage], stream), "cudaEventRecord");
        ++stage;
    };
    launch_ntt_forward(s.residues, s.primes, s.fwd, s.r, n, h.n_sub, h.split, stream);
    mark();
    launch_pointwise(s.residues, s.primes, s.zeta, s.r, n, h.n_sub, h.split, stream);
    mark();
    launch_ntt_inverse(s.residues, s.primes, s.inv, s.r, n, h.n_sub, h.split, stream);
    mark();
    launch_transpose(s.residues, s.crt_in, s.r, s.padded_r, n, h.n_sub, h.split, stream);
    mark();
}

// Enqueues the whole product on `stream`. `operands` already holds the padded inputs.
// `marks` (optional, kStages events) are recorded after each stage.
void enqueue_product(negacyclic_plan& s, uint32_t* d_c, cudaStream_t stream, cudaEvent_t* marks = nullptr) {
    const HostPlan& h = s.host;
    enqueue_convert(s, 0, h.n_sub, stream);
    if (marks) check(cudaEventRecord(marks[0], stream), "cudaEventRecord");
    enqueue_middle(s, stream, marks ? marks + 1 : nullptr);
    enqueue_output(s, 0, h.n, d_c, stream, marks ? marks[5] : nullptr);
    if (marks) check(cudaEventRecord(marks[6], stream), "cudaEventRecord");
    check(cudaGetLastError(), "product kernels");
}

int cuda_failure(const CudaError& e) {
    return fail(NEGACYCLIC_ECUDA, std::string(e.where) + ": " + cudaGetErrorString(e.code));
}

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

}  // namespace

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
    s.padded_limbs = round_up(limbs, 4);
    s.k_convert = 4 * s.padded_limbs;
    s.k_crt = 4 * s.padded_r;
    s.crt_columns = round_up(4 * h.words, 64);
    try {
        check(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaStreamCreateWithFlags(&s.copy_in, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaStreamCreateWithFlags(&s.copy_out, cudaStreamNonBlocking), "cudaStreamCreate");
        // host products stream in 8 coefficient chunks once each chunk keeps 128-row GEMM tiles
        s.chunks = (h.n_sub >= 1024 && h.n >= 8192) ? 8 : 1;
        for (uint32_t c = 0; c < s.chunks; ++c) {
            check(cudaEventCreateWithFlags(&s.in_ready[c], cudaEventDisableTiming), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&s.out_ready[c], cudaEventDisableTiming), "cudaEventCreate");
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
        device_alloc(s.crt_words, size_t(s.r) * h.words, work);
        device_alloc(s.operands, size_t(2) * n * s.padded_limbs, work);
        device_alloc(s.residues, size_t(2) * s.r * n, work);
        device_alloc(s.crt_in, size_t(n) * s.padded_r, work);
        device_alloc(s.dots, size_t(n) * h.words, work);
        device_alloc(s.result, size_t(n) * limbs, work);
        device_alloc(s.error_flag, 1, work);
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
        check(cudaMemcpyAsync(s.crt_words, h.crt_weights.data(), h.crt_weights.size() * 4, cudaMemcpyHostToDevice, st),
              "upload crt");
        check(cudaMemsetAsync(s.error_flag, 0, 4, st), "memset");
        // the K-padding columns of the operands stay zero forever
        check(cudaMemsetAsync(s.operands, 0, size_t(2) * n * s.padded_limbs * 4, st), "memset");
        launch_twiddles(s.primes, s.r, h.n_sub, s.fwd, s.inv, s.zeta, st);
        launch_convert_weights(s.primes, s.r, s.padded_r, limbs, s.k_convert, s.convert_weights, st);
        launch_crt_weights(s.crt_words, s.r, s.padded_r, h.words, s.crt_columns, s.crt_weights, st);
        check(cudaGetLastError(), "table kernels");
        check(cudaStreamSynchronize(st), "plan tables");

        if (o.gemm != NEGACYCLIC_GEMM_SIMT) {
            std::string why_convert, why_crt;
            if (prepare_gemm_tensor(s.convert_gemm, reinterpret_cast<const uint8_t*>(s.operands),
                                    uint64_t(s.padded_limbs) * 4, RowMap::split_rows(n, h.n_sub, h.split, 0, h.n_sub), 2 * n,
                                    s.convert_weights, 4 * s.padded_r, s.k_convert, why_convert))
                s.convert_engine = NEGACYCLIC_GEMM_TENSOR;
            if (prepare_gemm_tensor(s.crt_gemm, reinterpret_cast<const uint8_t*>(s.crt_in), uint64_t(s.padded_r) * 4,
                                    RowMap::linear(0), n, s.crt_weights, s.crt_columns,
                                    s.k_crt, why_crt))
                s.crt_engine = NEGACYCLIC_GEMM_TENSOR;
            if (o.gemm == NEGACYCLIC_GEMM_TENSOR &&
                (s.convert_engine != NEGACYCLIC_GEMM_TENSOR || s.crt_engine != NEGACYCLIC_GEMM_TENSOR))
                return fail(NEGACYCLIC_EINVAL, "tensor-core GEMM not available for this point: " + why_convert +
                                                   (why_convert.empty() ? "" : "; ") + why_crt);
        }
    } catch (const CudaError& e) {
        cudaGetLastError();
        return e.code == cudaErrorMemoryAllocation ? fail(NEGACYCLIC_ENOMEM, "device allocation failed")
                                                   : cuda_failure(e);
    }
    *out = plan.release();
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
    DeviceGuard guard(s->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    try {
        launch_pad_operands(d_a, d_b, s->operands, s->host.n, s->host.limbs, s->padded_limbs, stream);
        enqueue_product(*s, d_c, stream);
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

int negacyclic_run_device_timed(negacyclic_plan* s, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                                void* stream_ptr, float* stage_ms) {
    if (!s || !d_a || !d_b || !d_c || !stage_ms) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    DeviceGuard guard(s->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    cudaEvent_t events[kStages + 2] = {};
    int status = NEGACYCLIC_OK;
    try {
        for (auto& e : events) check(cudaEventCreate(&e), "cudaEventCreate");
        check(cudaEventRecord(events[0], stream), "cudaEventRecord");
        launch_pad_operands(d_a, d_b, s->operands, s->host.n, s->host.limbs, s->padded_limbs, stream);
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

int negacyclic_run(negacyclic_plan* s, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (!s || !a || !b || !c) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    DeviceGuard guard(s->device);
    const HostPlan& h = s->host;
    const size_t row = size_t(h.limbs) * 4, pitch = size_t(s->padded_limbs) * 4;
    const uint32_t chunks = s->chunks, per = h.n / chunks, span = h.n_sub / chunks;
    cudaStream_t st = s->stream;
    try {
        // inputs: chunk c's rows of a and b land in the padded operand layout (2-D copies, no pad
        // kernel), then the conversion GEMM of that chunk runs while the next chunk is in flight
        for (uint32_t k = 0; k < chunks; ++k) {
            const size_t first = size_t(k) * per;
            check(cudaMemcpy2DAsync(s->operands + first * s->padded_limbs, pitch, a + first * h.limbs, row, row, per,
                                    cudaMemcpyHostToDevice, s->copy_in),
                  "copy a");
            check(cudaMemcpy2DAsync(s->operands + (size_t(h.n) + first) * s->padded_limbs, pitch,
                                    b + first * h.limbs, row, row, per, cudaMemcpyHostToDevice, s->copy_in),
                  "copy b");
            check(cudaEventRecord(s->in_ready[k], s->copy_in), "cudaEventRecord");
            check(cudaStreamWaitEvent(st, s->in_ready[k], 0), "cudaStreamWaitEvent");
            enqueue_convert(*s, k * span, span, st);
        }
        enqueue_middle(*s, st, nullptr);
        // outputs: CRT GEMM + reduction per chunk, each chunk's copy-out overlapping the next chunk
        for (uint32_t k = 0; k <= chunks; ++k) {
            if (k < chunks) {
                enqueue_output(*s, k * per, per, s->result, st);
                check(cudaEventRecord(s->out_ready[k], st), "cudaEventRecord");
            }
            if (k >= 1) {
                const size_t first = size_t(k - 1) * per;
                check(cudaStreamWaitEvent(s->copy_out, s->out_ready[k - 1], 0), "cudaStreamWaitEvent");
                check(cudaMemcpyAsync(c + first * h.limbs, s->result + first * h.limbs, size_t(per) * row,
                                      cudaMemcpyDeviceToHost, s->copy_out),
                      "copy c");
            }
        }
        check(cudaGetLastError(), "product kernels");
        uint32_t flag = 0, pipeline = 0;
        check(cudaMemcpyAsync(&flag, s->error_flag, 4, cudaMemcpyDeviceToHost, s->copy_out), "error flag");
        if (uint32_t* tc = tensor_gemm_error_flag())
            check(cudaMemcpyAsync(&pipeline, tc, 4, cudaMemcpyDeviceToHost, s->copy_out), "error flag");
        check(cudaStreamSynchronize(s->copy_out), "product");
        check(cudaStreamSynchronize(st), "product");
        if (flag) return fail(NEGACYCLIC_ECUDA, "reduction exceeded its proven correction bound");
        if (pipeline) return fail(NEGACYCLIC_ECUDA, "tensor-core GEMM pipeline wait timed out");
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
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
    cudaError_t e = cudaMemcpy(host, src, size, cudaMemcpyDeviceToHost);
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
            launch_gemm_tensor(plan, raw, stream, rows, m, engine == NEGACYCLIC_GEMM_TENSOR);
        } else {
            launch_gemm_simt(d_a, k, rows, m, d_b, n, k, raw, stream);
        }
        check(cudaGetLastError(), "gemm");
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

}  // extern "C"
