/*
 * CPU ORACLE — test infrastructure only.
 *
 * Exact negacyclic product c = a*b mod (X^N + 1, q) over coefficient-major,
 * little-endian uint32 limbs, computed the way the reference's CPU checker
 * does it: Kronecker packing into one big integer, one GMP multiplication,
 * then "slot i minus slot i+N" and a reduction mod q.
 *
 * Restates tests/reference.py:29-43 (`kronecker`) of pokymono/fherma-polynomial-cuda:
 *   stride = ceil(bitlen(N*(q-1)^2) / 8) bytes per slot          (reference.py:37)
 *   left/right = little-endian concatenation of the slots         (reference.py:38-39)
 *   raw = left*right, c_i = (slot_i - slot_{i+N}) mod q            (reference.py:40-43)
 * and the schoolbook cross-check tests/reference.py:19-26 (`schoolbook`).
 *
 * The reference calls GMP through gmpy2, which is not installed here. The GMP
 * runtime (libgmp.so.10) is, but not its header, so the few mpz entry points
 * used are declared by hand below (their documented C signatures; mpz_t is the
 * documented {alloc, size, limb pointer} struct). Linked with -l:libgmp.so.10.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg may load this
 * library. Nothing in the product links it.
 */
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int alloc;
    int size;
    void* limbs;
} mpz_struct;
typedef mpz_struct mpz_t[1];

extern void __gmpz_init(mpz_struct*);
extern void __gmpz_clear(mpz_struct*);
extern void __gmpz_import(mpz_struct*, size_t count, int order, size_t size, int endian,
                          size_t nails, const void* op);
extern void* __gmpz_export(void* rop, size_t* countp, int order, size_t size, int endian,
                           size_t nails, const mpz_struct* op);
extern void __gmpz_mul(mpz_struct*, const mpz_struct*, const mpz_struct*);
extern void __gmpz_add(mpz_struct*, const mpz_struct*, const mpz_struct*);
extern void __gmpz_sub(mpz_struct*, const mpz_struct*, const mpz_struct*);
extern void __gmpz_sub_ui(mpz_struct*, const mpz_struct*, unsigned long);
extern void __gmpz_mul_ui(mpz_struct*, const mpz_struct*, unsigned long);
extern void __gmpz_fdiv_r(mpz_struct*, const mpz_struct*, const mpz_struct*);
extern size_t __gmpz_sizeinbase(const mpz_struct*, int base);
extern int __gmpz_cmp(const mpz_struct*, const mpz_struct*);
extern void __gmpz_set_ui(mpz_struct*, unsigned long);

/* limbs (little-endian uint32) -> mpz */
static void load_limbs(mpz_struct* z, const uint32_t* limbs, size_t count) {
    __gmpz_import(z, count, -1, sizeof(uint32_t), 0, 0, limbs);
}

/* mpz (non-negative, < 2^(32*count)) -> limbs, zero-filled */
static void store_limbs(uint32_t* limbs, size_t count, const mpz_struct* z) {
    size_t written = 0;
    memset(limbs, 0, count * sizeof(uint32_t));
    if (z->size == 0) return;
    /* export may write at most count words: the caller guarantees z < q < 2^(32*count) */
    __gmpz_export(limbs, &written, -1, sizeof(uint32_t), 0, 0, z);
}

/* ceil(bitlen(N*(q-1)^2) / 8), the slot width of reference.py:37 */
size_t oracle_slot_bytes(uint32_t n, uint32_t limbs, const uint32_t* q) {
    mpz_t zq, bound;
    __gmpz_init(zq);
    __gmpz_init(bound);
    load_limbs(zq, q, limbs);
    __gmpz_sub_ui(zq, zq, 1);
    __gmpz_mul(bound, zq, zq);
    __gmpz_mul_ui(bound, bound, n);
    size_t bits = bound->size == 0 ? 0 : __gmpz_sizeinbase(bound, 2);
    __gmpz_clear(zq);
    __gmpz_clear(bound);
    return (bits + 7) / 8;
}

/* Packs n coefficients of `limbs` words each into n slots of `stride` bytes. */
static void pack(mpz_struct* z, const uint32_t* x, uint32_t n, uint32_t limbs, size_t stride) {
    size_t total = (size_t)n * stride;
    unsigned char* buffer = (unsigned char*)calloc(total ? total : 1, 1);
    size_t coefficient_bytes = (size_t)limbs * 4;
    size_t copy = coefficient_bytes < stride ? coefficient_bytes : stride;
    for (uint32_t i = 0; i < n; ++i)
        memcpy(buffer + (size_t)i * stride, (const unsigned char*)(x + (size_t)i * limbs), copy);
    __gmpz_import(z, total, -1, 1, 0, 0, buffer);
    free(buffer);
}

/*
 * c = a*b mod (X^n + 1, q). a, b, c: [n][limbs] uint32, little-endian limbs.
 * Inputs must be canonical (< q). Returns 0, or -1 when q is zero.
 */
int oracle_negacyclic_kronecker(uint32_t n, uint32_t limbs, const uint32_t* q,
                                const uint32_t* a, const uint32_t* b, uint32_t* c) {
    mpz_t zq, left, right, product, hi, lo;
    __gmpz_init(zq);
    load_limbs(zq, q, limbs);
    if (zq->size == 0) {
        __gmpz_clear(zq);
        return -1;
    }
    size_t stride = oracle_slot_bytes(n, limbs, q);
    if (stride == 0) stride = 1; /* q == 1: every product slot is zero */
    __gmpz_init(left);
    __gmpz_init(right);
    __gmpz_init(product);
    __gmpz_init(hi);
    __gmpz_init(lo);
    pack(left, a, n, limbs, stride);
    pack(right, b, n, limbs, stride);
    __gmpz_mul(product, left, right);
    __gmpz_clear(left);
    __gmpz_clear(right);

    size_t raw_bytes = 2 * (size_t)n * stride;
    unsigned char* raw = (unsigned char*)calloc(raw_bytes, 1);
    size_t written = 0;
    if (product->size) __gmpz_export(raw, &written, -1, 1, 0, 0, product);
    __gmpz_clear(product);
    for (uint32_t i = 0; i < n; ++i) {
        __gmpz_import(lo, stride, -1, 1, 0, 0, raw + (size_t)i * stride);
        __gmpz_import(hi, stride, -1, 1, 0, 0, raw + ((size_t)i + n) * stride);
        __gmpz_sub(lo, lo, hi);
        __gmpz_fdiv_r(lo, lo, zq); /* floor remainder: 0 <= lo < q */
        store_limbs(c + (size_t)i * limbs, limbs, lo);
    }
    free(raw);
    __gmpz_clear(hi);
    __gmpz_clear(lo);
    __gmpz_clear(zq);
    return 0;
}

/*
 * Schoolbook negacyclic product (tests/reference.py:19-26), for small n.
 * Also used to spot-check single output coefficients of large products:
 * `first`..`first+count-1` are the coefficients computed (the rest untouched).
 */
int oracle_negacyclic_schoolbook(uint32_t n, uint32_t limbs, const uint32_t* q,
                                 const uint32_t* a, const uint32_t* b, uint32_t* c,
                                 uint32_t first, uint32_t count) {
    mpz_t zq, acc, x, y, t;
    __gmpz_init(zq);
    load_limbs(zq, q, limbs);
    if (zq->size == 0) {
        __gmpz_clear(zq);
        return -1;
    }
    __gmpz_init(acc);
    __gmpz_init(x);
    __gmpz_init(y);
    __gmpz_init(t);
    for (uint32_t k = first; k < first + count && k < n; ++k) {
        __gmpz_set_ui(acc, 0);
        for (uint32_t i = 0; i < n; ++i) {
            /* j with i + j == k (mod n); wrapping past n negates */
            uint32_t j = (k >= i) ? k - i : k + n - i;
            load_limbs(x, a + (size_t)i * limbs, limbs);
            load_limbs(y, b + (size_t)j * limbs, limbs);
            __gmpz_mul(t, x, y);
            if (k >= i)
                __gmpz_add(acc, acc, t);
            else
                __gmpz_sub(acc, acc, t);
        }
        __gmpz_fdiv_r(acc, acc, zq);
        store_limbs(c + (size_t)k * limbs, limbs, acc);
    }
    __gmpz_clear(acc);
    __gmpz_clear(x);
    __gmpz_clear(y);
    __gmpz_clear(t);
    __gmpz_clear(zq);
    return 0;
}
