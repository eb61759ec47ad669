/*
 * negacyclic.h — C ABI of the B200 exact negacyclic product
 *
 *     c = a * b  mod (X^N + 1, q)
 *
 * Operands and result are coefficient-major arrays of N coefficients, each L
 * little-endian uint32 limbs (limb j of coefficient i at index i*L + j), the
 * layout of the reference's fherma::Tensor<uint32_t> with shape {N, L}
 * (src/fherma.h:16-41). Inputs must be canonical (every coefficient < q); the
 * result is canonical.
 *
 * These entry points replace the reference's plugin entry points
 *   fherma_init  (src/fherma.h:46)  -> negacyclic_init
 *   fherma_run   (src/fherma.h:47)  -> negacyclic_run / negacyclic_run_device
 *   fherma_free  (src/fherma.h:48)  -> negacyclic_free
 * with plain pointers and sizes instead of C++ containers, and status codes
 * plus a thread-local message instead of exceptions (the reference throws
 * std::runtime_error, src/solve.cu:32-34, 506-507, 579). The fherma_* C++
 * entry points themselves are provided on top of this ABI by
 * libfherma_negacyclic.so (include/fherma_b200.h).
 *
 * Threading: one plan is not re-entrant — calls on the same plan must not
 * overlap. Distinct plans are independent.
 */
#ifndef NEGACYCLIC_H
#define NEGACYCLIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define NEGACYCLIC_OK 0
#define NEGACYCLIC_EINVAL 1     /* invalid point or argument (src/solve.cu:506-507) */
#define NEGACYCLIC_ENOFIELDS 2  /* not enough NTT primes for the bound (src/solve.cu:513) */
#define NEGACYCLIC_ESIZE 3      /* wrong operand size (src/solve.cu:579) */
#define NEGACYCLIC_ECUDA 4      /* a CUDA runtime/driver call failed (src/solve.cu:32-34) */
#define NEGACYCLIC_ENOMEM 5     /* device or pinned host allocation failed */
#define NEGACYCLIC_ENODEV 6     /* no usable sm_100 device */
#define NEGACYCLIC_EBUSY 7      /* serving form: the request queue is full; the request was not taken */

/* Bits of a plan's device status word (negacyclic_plan_status, negacyclic_batch_status). The
 * reference has no device-side error word: its waits are unbounded and its reduction has no
 * bound to exceed (src/solve.cu:468-490). */
#define NEGACYCLIC_STATUS_REDUCE 0x1u           /* a coefficient needed more corrections than proven */
#define NEGACYCLIC_STATUS_GEMM_MASK 0x1ffff00u  /* a tensor-core GEMM pipeline wait gave up (which role: bits) */

/* GEMM engine for the two byte-sliced products (conversion and CRT). */
#define NEGACYCLIC_GEMM_AUTO 0   /* tensor cores where the shape allows it */
#define NEGACYCLIC_GEMM_SIMT 1   /* dp4a CUDA-core kernel (any shape) */
#define NEGACYCLIC_GEMM_TENSOR 2 /* tcgen05 kind::i8, TMA-fed, TMEM accumulators (CTA pairs where possible) */
#define NEGACYCLIC_GEMM_TENSOR_SINGLE 3 /* tcgen05 with single-CTA 128x256 tiles only (no CTA pairs) */

typedef struct negacyclic_plan negacyclic_plan;

typedef struct {
    uint32_t split;     /* ring split s (power of two); 0 = smallest that works */
    uint32_t gemm;      /* NEGACYCLIC_GEMM_* */
    int32_t device;     /* CUDA device ordinal; -1 = the calling thread's current device */
    uint32_t external_work; /* 1: allocate no work space; bind one with negacyclic_bind_work */
    uint32_t reserved[4];
} negacyclic_options;

typedef struct {
    uint32_t n, w, limbs;     /* the point */
    uint32_t primes;          /* r: number of 31-bit NTT primes */
    uint32_t padded_primes;   /* r rounded up for the CRT GEMM's K dimension */
    uint32_t split;           /* s */
    uint32_t n_sub;           /* N' = N / s, the NTT length */
    uint32_t words;           /* words of the CRT sum: L + 5 */
    uint32_t gemm;            /* tensor-core use: bit 0 conversion GEMM, bit 1 CRT GEMM (0 = both SIMT) */
    uint32_t q_bits;          /* bit length of q */
    uint64_t device_bytes;    /* device memory held by the plan */
    uint64_t table_bytes;     /* of which parameter-only tables */
    uint32_t kernels_per_product; /* kernel launches of one negacyclic_run_device call */
    uint32_t reserved;
} negacyclic_info;

/* Message of the last failed call on this thread ("" if none). */
const char* negacyclic_last_error(void);

/*
 * Builds a plan for one point: picks primes p = 1 (mod 2N/s) in [2^30, 2^31)
 * with product P > 4N(q-1)^2, and uploads twiddle, conversion and CRT tables.
 * n: power of two, 1 <= n <= 131072. w: bit width with limbs == (w + 31) / 32
 * (src/solve.cu:506). q: `limbs` words, q >= 2. Parameter-only: no operand
 * data is touched. opts may be NULL.
 */
int negacyclic_init(uint32_t n, uint32_t w, uint32_t limbs, const uint32_t* q,
                    const negacyclic_options* opts, negacyclic_plan** plan);

/* Fills *info. */
int negacyclic_get_info(const negacyclic_plan* plan, negacyclic_info* info);

/*
 * Host-to-host product: a, b, c are host arrays of n*limbs words (c may alias
 * neither input). Copies in, computes, copies out; returns when c is written.
 * Streamed in chunks: copies of chunk k+1 overlap the conversion of chunk k on
 * the way in (rows of 1 KB or more go transform by transform, so each transform's
 * forward NTTs also overlap later copies), and the CRT/reduction of chunk k+1
 * overlaps the copy-out of chunk k on the way out. Page-locked host memory (cudaHostAlloc /
 * cudaHostRegister) is read and written by DMA directly; pageable memory goes
 * through the plan's page-locked staging buffers, filled and drained by a team of
 * host threads.
 */
int negacyclic_run(negacyclic_plan* plan, const uint32_t* a, const uint32_t* b, uint32_t* c);

/* Allocates now the page-locked staging and host copy threads that negacyclic_run
 * otherwise makes on its first call with pageable arrays (3 N L words pinned), and
 * runs one product of zero operands through the host path, so that the first real
 * call does not pay for loading kernels or first use of the staging pages. Depends
 * on the parameters only. */
int negacyclic_prepare_host(negacyclic_plan* plan);

/*
 * negacyclic_run in two halves, so that a caller can do host work (such as
 * allocating the output array) while the device computes: begin enqueues
 * everything with the result staged in page-locked memory (pageable inputs are
 * packed into staging by the plan's host threads, each chunk handed to the copy
 * engine as soon as it is packed); finish waits and has the host threads copy
 * each output chunk into c as it lands. a and b must stay valid until finish
 * returns.
 */
int negacyclic_run_begin(negacyclic_plan* plan, const uint32_t* a, const uint32_t* b);
int negacyclic_run_finish(negacyclic_plan* plan, uint32_t* c);

/*
 * Writes zeros over host memory [ptr, ptr + bytes) with the plan's host threads, so
 * that the first touch of a freshly allocated output array (page faults and the
 * kernel's zeroing, about 0.35 ms per MB on one core) is paid by all of them at
 * once. For callers that must allocate a new output array per product, as the
 * reference's fherma_run does (src/solve.cu:611); call it between run_begin and
 * run_finish, while the device computes. Blocking.
 */
int negacyclic_host_touch(negacyclic_plan* plan, void* ptr, size_t bytes);

/*
 * Device-resident product: d_a, d_b, d_c are device arrays of n*limbs words on
 * the plan's device. Enqueued on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) and returns without waiting. Device-side failures (a GEMM
 * pipeline wait that gave up, a reduction beyond its proven bound) set bits in
 * the plan's status word, which negacyclic_plan_status reads.
 */
int negacyclic_run_device(negacyclic_plan* plan, const uint32_t* d_a, const uint32_t* d_b,
                          uint32_t* d_c, void* stream);

/*
 * negacyclic_run_device, synchronously, with CUDA events recorded on `stream`
 * between stages. stage_ms[8] receives the milliseconds of: pad, convert,
 * forward NTT, pointwise, inverse NTT, transpose, CRT GEMM, reduce.
 */
int negacyclic_run_device_timed(negacyclic_plan* plan, const uint32_t* d_a, const uint32_t* d_b,
                                uint32_t* d_c, void* stream, float* stage_ms);

/*
 * Waits for the plan's device (cudaDeviceSynchronize), then stores the plan's
 * status word in *flags (NEGACYCLIC_STATUS_* bits; 0 = every product since the
 * last read was sound) and clears it. The device entry points, including
 * negacyclic_run_device_static, only ever set bits in the word; negacyclic_run
 * clears it when it starts and fails with NEGACYCLIC_ECUDA when it ends nonzero.
 */
int negacyclic_plan_status(negacyclic_plan* plan, uint32_t* flags);

/* Bytes of device work space one product of this plan needs (operands, residues, CRT
 * inputs and word sums, result). */
size_t negacyclic_work_bytes(const negacyclic_plan* plan);

/*
 * Binds a caller-owned, 256-byte-aligned device work space of at least
 * negacyclic_work_bytes() bytes to a plan created with external_work = 1.
 * Several plans may share one work space when their products never overlap
 * in time (same stream); products in flight on different streams need
 * different work spaces.
 */
int negacyclic_bind_work(negacyclic_plan* plan, void* d_work, size_t bytes);

/*
 * No counterpart in the reference: an addition of this library for callers that
 * cannot allocate device memory while they run (cudaFree waits for the whole
 * device; a framework's allocator may hold nearly all of HBM; a host process may
 * forbid allocations after start-up).
 *
 * negacyclic_run_device without allocation: the same product, enqueued on
 * `stream`, with the work space in a static device array of
 * NEGACYCLIC_STATIC_WORK_BYTES that the library keeps on each GPU it runs on.
 * Make the plan at start-up with external_work = 1 (tables only). Points whose
 * negacyclic_work_bytes() exceeds the array are rejected (NEGACYCLIC_EINVAL, the
 * message names both sizes); 64 MiB holds e.g. N = 8192 with L = 128. The plan's
 * own work-space binding is left as it was. Device-side errors go to the plan's
 * status word (negacyclic_plan_status), which lives with the plan's tables.
 * The first call on a device looks up the array's address (and makes the driver
 * load it); make that first call before any stream capture. Under
 * CUDA_MODULE_LOADING=EAGER the driver instead loads it, and so reserves the
 * 64 MiB, on every device when the process's context is created, whether or not
 * this entry point is called. All calls share the array: calls whose work
 * overlaps on the GPU (other streams, unordered threads) race and corrupt each
 * other, so order them on one stream or with events.
 */
#define NEGACYCLIC_STATIC_WORK_BYTES ((size_t)64 << 20)
int negacyclic_run_device_static(negacyclic_plan* plan, const uint32_t* d_a, const uint32_t* d_b,
                                 uint32_t* d_c, void* stream);

/*
 * Diagnostics of the current device: *flags receives the device-wide tensor-core
 * GEMM word (nonzero = a pipeline wait of any GEMM gave up since the last call;
 * bits say which role) and the word is cleared. Synchronises the device. Each
 * product also reports its own failures in its plan's status word.
 */
int negacyclic_pipeline_status(uint32_t* flags);

/*
 * Diagnostic of the tensor-core GEMM's failure path, with no counterpart in the
 * reference (its waits have no bound). Runs the raw GEMM of negacyclic_gemm_u8
 * (engine NEGACYCLIC_GEMM_TENSOR or _TENSOR_SINGLE) with every pipeline wait
 * bounded by limit_cycles of SM clock, on a stream of its own, and with the TMA
 * producer of the first CTA (pair) stopping before pipeline step withheld_step
 * (0xffffffff: never), so that the stage its MMA issuer waits for never arrives.
 * The wait runs out, every role of that CTA (pair) stops, and the kernel returns;
 * *flags receives the status word (NEGACYCLIC_STATUS_GEMM_MASK bits) and
 * *elapsed_ms the kernel's device time. Returns NEGACYCLIC_ECUDA when flags is
 * nonzero. Blocking. d_d is left partly unwritten on failure.
 */
int negacyclic_gemm_u8_withheld(const uint8_t* d_a, const uint8_t* d_b, int32_t* d_d, uint32_t m, uint32_t n,
                                uint32_t k, uint32_t engine, uint64_t limit_cycles, uint32_t withheld_step,
                                uint32_t* flags, double* elapsed_ms);

/* Releases the plan and every device/pinned buffer it holds. NULL is a no-op. */
void negacyclic_free(negacyclic_plan* plan);

/*
 * Host-only plan constants (no GPU needed), for checking the parameter
 * selection against an independent model. Arrays are caller-allocated:
 *   primes[r], finish[r] (F_k = 2^96 N'^-1 (P/p_k)^-1 mod p_k),
 *   crt_mod_q[r * limbs] (M_k = (P/p_k) mod q), minus_p_mod_q[limbs].
 * Pass max_primes = 0 to query r, s and N' only.
 */
int negacyclic_host_plan(uint32_t n, uint32_t limbs, const uint32_t* q, uint32_t split,
                         uint32_t max_primes, uint32_t* primes_out, uint32_t* split_out,
                         uint32_t* n_sub_out, uint32_t* primes, uint32_t* finish,
                         uint32_t* crt_mod_q, uint32_t* minus_p_mod_q);

/*
 * Copies one internal stage buffer of the last product to host memory, for
 * stage-by-stage checks at small sizes. which: 0 residues [2][r][N] u32 (after
 * the last stage that wrote them), 1 CRT inputs [N][padded_primes] u32,
 * 2 CRT word sums [N][words] u64. Returns the byte size in *bytes when host is NULL.
 */
int negacyclic_debug_read(negacyclic_plan* plan, int which, void* host, size_t* bytes);

/*
 * Raw u8 GEMM check: D[m][n] = sum_k A[m][k] * B[n][k] (int32) with both
 * engines, for testing the tensor-core kernel against the SIMT one.
 * A: [m][k] u8 device, B: [n][k] u8 device, D: [m][n] int32 device. k % 16 == 0.
 */
int negacyclic_gemm_u8(const uint8_t* d_a, const uint8_t* d_b, int32_t* d_d, uint32_t m,
                       uint32_t n, uint32_t k, uint32_t engine, void* stream);

/* ---------------------------------------------------------------------------
 * Batched form: many products of uneven (N, W, q) in one graph launch.
 * New in this library (the reference runs one product per harness call,
 * src/main.cpp:164-204). Instances are planned individually (an autotuner picks
 * each shape's ring split and GEMM kernel by timing them, cached in a text file)
 * and captured into a single CUDA graph. By default the graph has two phases:
 * instances under about 1 ms of device time share the GPU on up to four compute
 * lanes (single-CTA tensor GEMMs), then the larger ones run one after another on
 * lane 0 with CTA-pair GEMMs. lanes > 0 instead spreads every instance over that
 * many lanes. Each lane shares one work arena among its instances.
 */
typedef struct negacyclic_batch negacyclic_batch;

typedef struct {
    uint32_t n, w, limbs;  /* as for negacyclic_init */
    const uint32_t* q;     /* limbs words (read during negacyclic_batch_create only) */
} negacyclic_point;

typedef struct {
    uint32_t lanes;          /* 0 = two phases (see above); else every instance on this many streams
                                (single-CTA GEMM tiles when more than one) */
    uint32_t tune;           /* 1: time candidate configurations for shapes not in the cache */
    int32_t device;          /* -1 = current device */
    uint32_t reserved0;
    const char* tune_cache;  /* cache file; NULL = $NEGACYCLIC_TUNE_CACHE, or no cache */
    uint32_t reserved[4];
} negacyclic_batch_options;

typedef struct {
    negacyclic_info plan;    /* the instance's plan (split, primes, GEMM engines ...) */
    uint32_t lane;           /* stream it runs on */
    uint32_t requested_gemm; /* NEGACYCLIC_GEMM_* chosen by the tuner (0 = default) */
    double tuned_ms;         /* measured device time of one product (0 = not tuned) */
    uint32_t phase;          /* 0: runs concurrently with others; 1: runs alone, after phase 0 */
    uint32_t reserved;
} negacyclic_batch_instance;

int negacyclic_batch_create(const negacyclic_point* points, uint32_t count,
                            const negacyclic_batch_options* opts, negacyclic_batch** batch);

/* Device buffers of instance `index` ([N][L] words each): fill a and b, read c. */
int negacyclic_batch_io(negacyclic_batch* batch, uint32_t index, uint32_t** d_a, uint32_t** d_b,
                        uint32_t** d_c);

int negacyclic_batch_get_info(const negacyclic_batch* batch, uint32_t index,
                              negacyclic_batch_instance* info);

/* Every product of the batch from its device buffers: one cudaGraphLaunch on `stream`. The
 * graph first clears every instance's status word; read them with negacyclic_batch_status. */
int negacyclic_batch_run_device(negacyclic_batch* batch, void* stream);

/* Waits for the device, then stores each instance's status word in flags[0..count) (0 = sound;
 * NEGACYCLIC_STATUS_* bits otherwise) and clears them. */
int negacyclic_batch_status(negacyclic_batch* batch, uint32_t* flags);

/* Instance `index` alone, as one plain product (the per-call path), enqueued on `stream`.
 * Must not overlap other runs of the same batch (instances share lane work spaces). */
int negacyclic_batch_run_one(negacyclic_batch* batch, uint32_t index, void* stream);

/* Host arrays a[i], b[i], c[i] per instance: copy-in, compute and copy-out streams overlap
 * (instance i computes while later operands copy in and earlier results copy out). Blocking;
 * fails with NEGACYCLIC_ECUDA, naming the instance, when an instance's status word is set. */
int negacyclic_batch_run(negacyclic_batch* batch, const uint32_t* const* a, const uint32_t* const* b,
                         uint32_t* const* c);

/* The same host arrays one instance after another through negacyclic_run (the plain
 * per-call host path), for comparison. Blocking. */
int negacyclic_batch_run_plain(negacyclic_batch* batch, const uint32_t* const* a,
                               const uint32_t* const* b, uint32_t* const* c);

void negacyclic_batch_free(negacyclic_batch* batch);

/* ---------------------------------------------------------------------------
 * Serving form: a request loop with continuous batching (new in this library).
 * A session fixes (W, L, q); its plans, one per ring size N, stay resident on
 * the device. Requests are submitted from any thread and return at once; a
 * dispatcher admits them in arrival order whenever a stream slot is free and
 * their device memory fits the HBM budget, so work of requests that arrive
 * while others run overlaps on the device. Host buffers must stay valid until
 * negacyclic_server_wait returns; page-locked buffers overlap best.
 */
typedef struct negacyclic_server negacyclic_server;

typedef struct {
    uint64_t hbm_budget;  /* bytes for resident plan tables + in-flight requests; 0 = 60 GiB */
    uint32_t slots;       /* concurrent requests (streams); 0 = 4 */
    int32_t device;       /* -1 = current device */
    uint32_t max_queue;   /* requests waiting for admission beyond which submit refuses new ones
                             (NEGACYCLIC_EBUSY); 0 = no limit */
    uint32_t reserved[3];
} negacyclic_server_options;

typedef struct {
    uint64_t completed, failed, queued;
    uint64_t resident_bytes, in_flight_bytes;
    double p50_ms, p99_ms, mean_ms;  /* submit -> result on the host, completed requests */
    double products_per_s;           /* completed / (last finish - first submit) */
    uint64_t rejected;               /* submits refused because the queue was full */
    uint64_t max_queued;             /* deepest the admission queue has been */
} negacyclic_server_stats;

int negacyclic_server_create(const negacyclic_server_options* opts, negacyclic_server** server);

/* Opens a session for (W, L, q); plans for the `count` ring sizes in ns are built now
 * (others on their first request). The first request that launches a given kernel instance
 * (for instance the first of a new ring size) also loads that kernel's module, which costs tens
 * of milliseconds. A latency-sensitive caller sends one request per (session, N) before serving,
 * or sets CUDA_MODULE_LOADING=EAGER to load every module when the library is first used. */
int negacyclic_server_open_session(negacyclic_server* server, uint32_t w, uint32_t limbs,
                                   const uint32_t* q, const uint32_t* ns, uint32_t count,
                                   uint32_t* session);

/* Queues a request and returns at once; NEGACYCLIC_EBUSY (nothing queued) when max_queue requests
 * already wait for admission. */
int negacyclic_server_submit(negacyclic_server* server, uint32_t session, uint32_t n,
                             const uint32_t* a, const uint32_t* b, uint32_t* c, uint64_t* request);

/* Blocks until the request finished (or timeout_ms passed; <= 0 waits without limit). A request
 * whose product set its plan's status word fails with NEGACYCLIC_ECUDA. */
int negacyclic_server_wait(negacyclic_server* server, uint64_t request, double timeout_ms,
                           double* latency_ms);

int negacyclic_server_get_stats(negacyclic_server* server, negacyclic_server_stats* stats);

/* Stops the dispatcher after in-flight work finishes and frees everything. */
void negacyclic_server_free(negacyclic_server* server);

#ifdef __cplusplus
}
#endif

#endif /* NEGACYCLIC_H */
