// Device kernels of the negacyclic product (SIMT stages and table builders).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "modarith.cuh"

namespace negacyclic {

// Row addressing of the u8 GEMM's A operand, for one launch (a whole product or a chunk).
//  kRowsLinear: GEMM row m reads operand row first + m.
//  kRowsSplit:  GEMM row m = (op - op_first)*(t_count*span) + (t - t_first)*span + (j - first),
//               t in [t_first, t_first + t_count), j in [first, first + span), covers
//               coefficient i = s*j + t of operand op, which the pad kernels store
//               split-major at operand row op*N + t*N' + j, and produces residue row op,
//               column t*N' + j (transform t, position j). A (op, t) slab of rows is
//               contiguous, so every 128-row A tile is one plain 2-D box.
enum RowMode : int { kRowsLinear = 0, kRowsSplit = 1 };

struct RowMap {
    int mode;
    uint32_t n, n_sub, split;
    uint32_t first;    // linear: first operand row; split: first j
    uint32_t span;     // split: j values per (operand, t) in this launch
    uint32_t t_first;  // split: transforms [t_first, t_first + t_count) in this launch
    uint32_t t_count;
    uint32_t op_first = 0;  // split: first operand (0: a, 1: b); m / (t_count*span) operands

    static RowMap linear(uint32_t first_row) { return RowMap{kRowsLinear, 0, 0, 1, first_row, 0, 0, 1}; }
    static RowMap split_rows(uint32_t n, uint32_t n_sub, uint32_t split, uint32_t first_j, uint32_t j_span,
                             uint32_t t_first, uint32_t t_count, uint32_t op_first = 0) {
        return RowMap{kRowsSplit, n, n_sub, split, first_j, j_span, t_first, t_count, op_first};
    }
    __host__ __device__ __forceinline__ void decompose(uint32_t m, uint32_t& op, uint32_t& t, uint32_t& j) const {
        const uint32_t per_op = t_count * span, local_op = m / per_op;
        op = op_first + local_op;
        const uint32_t rem = m - local_op * per_op;
        const uint32_t dt = rem / span;
        t = t_first + dt;
        j = first + (rem - dt * span);
    }
    // operand row read by GEMM row m
    __device__ __forceinline__ uint64_t row(uint32_t m) const {
        if (mode == kRowsLinear) return uint64_t(first) + m;
        uint32_t op, t, j;
        decompose(m, op, t, j);
        return uint64_t(op) * n + uint64_t(t) * n_sub + j;
    }
    // conversion output position of GEMM row m: residue row `op`, column t*N' + j
    __device__ __forceinline__ void residue(uint32_t m, uint32_t& op, uint32_t& column) const {
        uint32_t t, j;
        decompose(m, op, t, j);
        column = t * n_sub + j;
    }
};

// Epilogues of the byte-sliced GEMM. Output column group g (4 consecutive
// columns 4g..4g+3) of row m holds int32 dots G_d; S = sum_d G_d 256^d.
enum EpilogueMode : int { kEpilogueRaw = 0, kEpilogueConvert = 1, kEpilogueCrt = 2 };

struct Epilogue {
    int mode;
    // raw: D[row][col] int32, ld = columns, row = the operand row of GEMM row m
    int32_t* raw;
    uint32_t raw_ld;
    // convert: residues[(op*r + k)*N + column] = redc(S, p_k), (op, column) = RowMap::residue(m), g = k < r
    uint32_t* residues;
    const DevicePrime* primes;
    uint32_t r, n;
    // crt: dots[row * dots_stride + g] = S (u64), g < words, row = the operand row of GEMM row m;
    //      dots_stride is words rounded up to a multiple of 8 (64-byte rows)
    uint64_t* dots;
    uint32_t words, dots_stride;
    // every mode: the product's status word (NEGACYCLIC_STATUS_*); the tensor-core kernels set
    // NEGACYCLIC_STATUS_GEMM_MASK bits in it when a pipeline wait gives up (nullptr: none kept)
    uint32_t* status;
};

// a, b: [N][L] -> out: [2][N][Lp], rows split-major (coefficient s*j + t at row op*N + t*N' + j),
// limbs padded with zeros to Lp
void launch_pad_operands(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n,
                         uint32_t limbs, uint32_t padded_limbs, uint32_t split, cudaStream_t stream);
// rows [first_row, first_row + count) of operands [op_first, op_first + op_count) (operand stride N
// rows) from an unpadded [2][N][L] array into the padded split-major [2][N][Lp] layout: staged in
// coefficient order (split = s, rows are permuted) or already split-major (split = 1)
void launch_pad_rows(const uint32_t* staged, uint32_t* out, uint32_t n, uint32_t limbs, uint32_t padded_limbs,
                     uint32_t split, uint32_t first_row, uint32_t count, cudaStream_t stream, uint32_t op_first = 0,
                     uint32_t op_count = 2);
void launch_twiddles(const DevicePrime* primes, uint32_t r, uint32_t n_sub, uint2* fwd, uint2* inv,
                     uint2* zeta, cudaStream_t stream);
void launch_convert_weights(const DevicePrime* primes, uint32_t r, uint32_t padded_r, uint32_t limbs,
                            uint32_t k_bytes, uint8_t* out, cudaStream_t stream);
void launch_crt_weights(const uint32_t* weights_words, uint32_t r, uint32_t padded_r, uint32_t words,
                        uint32_t columns, uint8_t* out, cudaStream_t stream);
void launch_gemm_simt(const uint8_t* a, uint64_t a_pitch, RowMap rows, uint32_t m, const uint8_t* b,
                      uint32_t columns, uint32_t k_bytes, const Epilogue& epilogue, cudaStream_t stream);
// forward NTTs of transforms [t_first, t_first + t_count) of operands [op_first, op_first + op_count),
// every prime
void launch_ntt_forward(uint32_t* residues, const DevicePrime* primes, const uint2* fwd, uint32_t r,
                        uint32_t n, uint32_t n_sub, uint32_t t_first, uint32_t t_count, cudaStream_t stream,
                        uint32_t op_first = 0, uint32_t op_count = 2);
void launch_pointwise(uint32_t* residues, const DevicePrime* primes, const uint2* zeta, uint32_t r,
                      uint32_t n, uint32_t n_sub, uint32_t split, cudaStream_t stream);
// inverse NTTs of transforms [v_first, v_first + v_count), every prime
void launch_ntt_inverse(uint32_t* residues, const DevicePrime* primes, const uint2* inv, uint32_t r,
                        uint32_t n, uint32_t n_sub, uint32_t v_first, uint32_t v_count, cudaStream_t stream);
// crt_in[s*j + v][k] = residues[0][k][v*N' + j] for every v and j in [j_first, j_first + j_count):
// coefficients [s j_first, s (j_first + j_count)); zero for k in [r, r')
void launch_transpose(const uint32_t* residues, uint32_t* crt_in, uint32_t r, uint32_t padded_r,
                      uint32_t n, uint32_t split, uint32_t j_first, uint32_t j_count, cudaStream_t stream);

struct ReduceParams {
    const uint64_t* dots;     // [n][dots_stride], words used
    uint32_t* out;            // [n][limbs]
    const uint32_t* q;        // [limbs]
    const uint32_t* minus_p;  // [limbs]  (-P) mod q
    uint32_t n, limbs, words, dots_stride;
    int32_t top_shift;
    uint64_t mu_low;
    uint32_t* error_flag;     // set nonzero if a coefficient needed more corrections than proven
};
void launch_reduce(const ReduceParams& params, cudaStream_t stream);

}  // namespace negacyclic
