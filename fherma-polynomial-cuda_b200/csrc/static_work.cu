// negacyclic_run_device_static: the device-resident product with its work space in a
// fixed array that this library holds on every GPU it runs on, so the call allocates
// nothing.
//
// Who needs this: callers that cannot call cudaMalloc once they are running.
//  * cudaFree waits for the whole device, which stalls every other stream.
//  * A framework's caching allocator may already own nearly all of HBM, so a
//    fresh cudaMalloc fails.
//  * A plugin host may forbid allocations after start-up.
// Such callers make their plans at start-up with external_work = 1, which allocates
// only the parameter tables, and then multiply through this entry point.
//
// The work space (padded operands, residues, CRT inputs and word sums, the result
// staging and the GEMM tile counter) is g_static_work below: 64 MiB, enough for
// products up to about N = 8192 with L = 128, or N = 4096 with L = 256. A point whose
// work space is larger is rejected with an error that names both sizes.
//
// In host code g_static_work is only a stand-in for the array. Its device address
// comes from cudaGetSymbolAddress, called with the device current on the first call
// of this entry point on that device (and again if the device's context was made
// anew, e.g. after cudaDeviceReset). That first call loads this file's module and so
// sets aside the array, which stays until the process exits. Make that first call
// before any stream capture. Under CUDA_MODULE_LOADING=EAGER the driver loads the
// module, and sets aside the 64 MiB, on every device when the context is created,
// whether or not this entry point is ever called.
//
// Every call shares the one array and leaves its contents behind:
//  * nothing in it needs to start at zero: the GEMM tile counter is cleared before
//    each GEMM, and the status word that reports device-side errors belongs to the
//    plan (read it with negacyclic_plan_status);
//  * padding limbs and padding prime columns meet zero weights in the GEMMs, so
//    whatever they hold never reaches the result;
//  * two calls whose work overlaps on the GPU (different streams, or different host
//    threads without ordering between them) overwrite each other's intermediates and
//    return wrong products; order such calls on one stream or with events.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/negacyclic.h"
#include "plan_internal.h"

using namespace negacyclic;
using namespace negacyclic::detail;

namespace {

constexpr size_t kStaticWorkBytes = NEGACYCLIC_STATIC_WORK_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_work[kStaticWorkBytes];

std::mutex g_static_mutex;
void* g_static_address[kMaxDevices] = {};
unsigned long long g_static_context[kMaxDevices] = {};  // context the address belongs to

using CtxGetCurrent = CUresult (*)(CUcontext*);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (0 if the driver cannot tell): a context made
// anew for the device gets a new id, and the array's address must then be looked up again.
unsigned long long current_context_id() {
    static CtxGetCurrent get_current = nullptr;
    static CtxGetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult found{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrent>(fn);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetId>(fn);
    });
    CUcontext context = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&context) != CUDA_SUCCESS || !context ||
        get_id(context, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of g_static_work on `device`, which the caller has made current: looked up once
// per device and context.
void* static_work_address(int device) {
    std::lock_guard<std::mutex> lock(g_static_mutex);
    const unsigned long long context = current_context_id();
    if (!g_static_address[device] || context == 0 || context != g_static_context[device]) {
        void* ptr = nullptr;
        check(cudaGetSymbolAddress(&ptr, g_static_work), "cudaGetSymbolAddress(static work space)");
        g_static_address[device] = ptr;
        g_static_context[device] = context;
    }
    return g_static_address[device];
}

// The plan fields that bind_work rewrites, so the plan's own binding can be put back.
struct Binding {
    uint32_t *operands, *residues, *crt_in, *result;
    uint64_t* dots;
    uint32_t convert_engine, crt_engine;
    TensorGemmPlan convert_gemm, crt_gemm;

    explicit Binding(const negacyclic_plan& s)
        : operands(s.operands), residues(s.residues), crt_in(s.crt_in), result(s.result), dots(s.dots), convert_engine(s.convert_engine), crt_engine(s.crt_engine),
          convert_gemm(s.convert_gemm), crt_gemm(s.crt_gemm) {}

    void restore(negacyclic_plan& s) const {
        s.operands = operands;
        s.residues = residues;
        s.crt_in = crt_in;
        s.result = result;
        s.dots = dots;
        s.convert_engine = convert_engine;
        s.crt_engine = crt_engine;
        s.convert_gemm = convert_gemm;
        s.crt_gemm = crt_gemm;
    }
};

}  // namespace

extern "C" int negacyclic_run_device_static(negacyclic_plan* s, const uint32_t* d_a, const uint32_t* d_b,
                                            uint32_t* d_c, void* stream_ptr) {
    if (!s || !d_a || !d_b || !d_c) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (s->device < 0 || s->device >= kMaxDevices) return fail(NEGACYCLIC_ENODEV, "device ordinal out of range");
    if (s->work_bytes > kStaticWorkBytes)
        return fail(NEGACYCLIC_EINVAL, "this point needs " + std::to_string(s->work_bytes) +
                                           " bytes of work space; the static work space holds " +
                                           std::to_string(kStaticWorkBytes) + " bytes");
    DeviceGuard guard(s->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const Binding own(*s);
    int status = NEGACYCLIC_OK;
    try {
        void* arena = static_work_address(s->device);
        const std::string why = bind_work(*s, arena);
        if (!why.empty()) {
            own.restore(*s);
            return fail(NEGACYCLIC_EINVAL, why);
        }
        // kernel arguments (pointers, tensor maps) are copied at launch, so the plan's own
        // binding can be put back as soon as the product is enqueued
        enqueue_device_product(*s, d_a, d_b, d_c, stream);
    } catch (const CudaError& e) {
        status = cuda_failure(e);
    }
    own.restore(*s);
    return status;
}
