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

/* GEMM engine for the two byte-sliced products (conversion and CRT). */
#define NEGACYCLIC_GEMM_AUTO 0   /* tensor cores where the shape allows it */
#define NEGACYCLIC_GEMM_SIMT 1   /* dp4a CUDA-core kernel (any shape) */
#define NEGACYCLIC_GEMM_TENSOR 2 /* tcgen05 kind::i8, TMA-fed, TMEM accumulators (CTA pairs where possible) */
#define NEGACYCLIC_GEMM_TENSOR_SINGLE 3 /* negacyclic_gemm_u8 only: the single-CTA tcgen05 kernel */

typedef struct negacyclic_plan negacyclic_plan;

typedef struct {
    uint32_t split;     /* ring split s (power of two); 0 = smallest that works */
    uint32_t gemm;      /* NEGACYCLIC_GEMM_* */
    int32_t device;     /* CUDA device ordinal; -1 = the calling thread's current device */
    uint32_t reserved[5];
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
 * Page-locked host memory (cudaHostAlloc / cudaHostRegister) is copied by DMA
 * directly; pageable memory goes through the plan's pinned staging buffers.
 */
int negacyclic_run(negacyclic_plan* plan, const uint32_t* a, const uint32_t* b, uint32_t* c);

/*
 * Device-resident product: d_a, d_b, d_c are device arrays of n*limbs words on
 * the plan's device. Enqueued on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) and returns without waiting.
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

#ifdef __cplusplus
}
#endif

#endif /* NEGACYCLIC_H */
