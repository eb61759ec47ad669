// SIMT stages of the negacyclic product and the parameter-only table builders.
//
// Data layout in HBM (one plan, r primes, ring split s, N' = N/s):
//   operands   [2][N][Lp] u32      a then b, limbs padded to Lp = roundup(L, 32) (128-byte rows),
//                                  split-major: row op*N + t*N' + j holds coefficient s*j + t
//   residues   [2][r][N]  u32      per (operand, prime): s transforms of N' values,
//                                  transform t holds coefficients i = s*j + t at j
//   crt_in     [N][r']    u32      coefficient-major residues v_k (r' = roundup(r, 32))
//   dots       [N][L+5]   u64      word sums of the byte-sliced CRT product
//   twiddles   [r][N']    uint2    {w, floor(w 2^32/p)}: forward psi^brv(m), inverse psi^-brv(m),
//                                  zeta psi^(2 brv(m)+1) (evaluation point at output m)
#include "kernels.cuh"

#include <algorithm>
#include <type_traits>

namespace negacyclic {

namespace {

constexpr uint32_t kFull = 0xffffffffu;

// One padded row: Lp words (16-byte aligned) from `limbs` words, zeros above.
__device__ __forceinline__ void pad_row(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t limbs,
                                        uint32_t padded, uint32_t lane) {
    uint4* out = reinterpret_cast<uint4*>(dst);
    for (uint32_t c = lane; c < padded / 4; c += 32) {
        const uint32_t w = 4 * c;
        uint4 v;
        v.x = w < limbs ? src[w] : 0u;
        v.y = w + 1 < limbs ? src[w + 1] : 0u;
        v.z = w + 2 < limbs ? src[w + 2] : 0u;
        v.w = w + 3 < limbs ? src[w + 3] : 0u;
        out[c] = v;
    }
}

// [N][L] a and b -> [2][N][Lp] split-major: output row op*N + t*N' + j holds coefficient
// s*j + t of operand op. One warp per output row.
__global__ void pad_operands_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                    uint32_t* __restrict__ out, uint32_t n, uint32_t limbs, uint32_t padded,
                                    uint32_t log_split, uint32_t log_n_sub) {
    const uint32_t lane = threadIdx.x % 32, warps = gridDim.x * (blockDim.x / 32);
    const uint32_t n_sub_mask = (1u << log_n_sub) - 1;
    for (uint32_t w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; w < 2 * n; w += warps) {
        const uint32_t op = w >= n ? 1 : 0, row = w - op * n;
        const uint32_t i = ((row & n_sub_mask) << log_split) + (row >> log_n_sub);
        pad_row((op ? b : a) + size_t(i) * limbs, out + size_t(w) * padded, limbs, padded, lane);
    }
}

// Rows [first, first + count) of operands [op_first, op_first + op_count) (operand stride N rows)
// from an unpadded [2][N][L] array into the padded split-major layout. Staged rows are either
// already split-major (log_split = 0: row = position) or in coefficient order (row i goes to
// t*N' + j, i = s*j + t). One warp per row.
__global__ void pad_rows_kernel(const uint32_t* __restrict__ staged, uint32_t* __restrict__ out, uint32_t n,
                                uint32_t limbs, uint32_t padded, uint32_t log_split, uint32_t log_n_sub,
                                uint32_t first, uint32_t count, uint32_t op_first, uint32_t op_count) {
    const uint32_t lane = threadIdx.x % 32, warps = gridDim.x * (blockDim.x / 32);
    const uint32_t split_mask = (1u << log_split) - 1;
    for (uint32_t w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; w < op_count * count; w += warps) {
        const uint32_t local_op = w / count, op = op_first + local_op, i = first + (w - local_op * count);
        const uint32_t row = ((i & split_mask) << log_n_sub) + (i >> log_split);
        pad_row(staged + (size_t(op) * n + i) * limbs, out + (size_t(op) * n + row) * padded, limbs, padded, lane);
    }
}

__device__ __forceinline__ uint32_t bit_reverse(uint32_t x, uint32_t bits) {
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

__global__ void twiddles_kernel(const DevicePrime* __restrict__ primes, uint32_t r, uint32_t n_sub,
                                uint32_t log_n, uint2* fwd, uint2* inv, uint2* zeta) {
    uint32_t k = blockIdx.y;
    if (k >= r) return;
    const DevicePrime f = primes[k];
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n_sub; m += gridDim.x * blockDim.x) {
        uint32_t e = bit_reverse(m, log_n);
        uint32_t w_fwd = pow_mod(f.psi, e, f);
        uint32_t w_inv = pow_mod(f.psi, 2ull * n_sub - e, f);
        uint32_t w_zeta = pow_mod(f.psi, 2ull * e + 1, f);
        size_t at = size_t(k) * n_sub + m;
        fwd[at] = make_uint2(w_fwd, shoup_quotient(w_fwd, f.p));
        inv[at] = make_uint2(w_inv, shoup_quotient(w_inv, f.p));
        zeta[at] = make_uint2(w_zeta, shoup_quotient(w_zeta, f.p));
    }
}

// B_conv[4k+d][j] = byte_d(256^j mod p_k); zero for padded primes and j >= 4L.
__global__ void convert_weights_kernel(const DevicePrime* __restrict__ primes, uint32_t r,
                                       uint32_t padded_r, uint32_t limbs, uint32_t k_bytes,
                                       uint8_t* out) {
    uint32_t k = blockIdx.y;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < k_bytes; j += gridDim.x * blockDim.x) {
        uint32_t w = 0;
        if (k < r && j < 4 * limbs) w = pow_mod(256, j, primes[k]);
        for (uint32_t d = 0; d < 4; ++d) out[(size_t(k) * 4 + d) * k_bytes + j] = uint8_t(w >> (8 * d));
    }
}

// B_crt[c][4k+d] = byte_{c-d}(W_k), W_k given as `words` u32 words; zero outside.
__global__ void crt_weights_kernel(const uint32_t* __restrict__ weights, uint32_t r, uint32_t padded_r,
                                   uint32_t words, uint32_t columns, uint8_t* out) {
    uint32_t c = blockIdx.y;
    const uint32_t k_bytes = 4 * padded_r;
    for (uint32_t kd = blockIdx.x * blockDim.x + threadIdx.x; kd < k_bytes; kd += gridDim.x * blockDim.x) {
        uint32_t k = kd / 4, d = kd % 4;
        uint8_t value = 0;
        if (k < r && c < columns && c >= d) {
            uint32_t at = c - d;  // byte position within W_k
            if (at < 4 * words) value = uint8_t(weights[size_t(k) * words + at / 4] >> (8 * (at % 4)));
        }
        out[size_t(c) * k_bytes + kd] = value;
    }
}

// ---------------------------------------------------------------------------
// SIMT byte GEMM: D[m][c] = sum_j A[m][j] * B[c][j] with dp4a, 64x64 tiles,
// 256 threads, each thread a 4-row x 4-column (one column group) micro-tile.
constexpr int kTile = 64, kTileK = 64;

__global__ void __launch_bounds__(256) gemm_simt_kernel(const uint8_t* __restrict__ a, uint64_t a_pitch,
                                                        RowMap rows, uint32_t m_total,
                                                        const uint8_t* __restrict__ b, uint32_t columns,
                                                        uint32_t k_bytes, Epilogue epi) {
    __shared__ uint32_t as[kTile][kTileK / 4 + 1];
    __shared__ uint32_t bs[kTile][kTileK / 4 + 1];
    const uint32_t tid = threadIdx.x, tr = tid / 16, tc = tid % 16;
    const uint32_t m0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
    const uint32_t load_row = tid / 4, load_part = tid % 4;
    const uint32_t am = m0 + load_row, bc = c0 + load_row;
    const uint8_t* arow = am < m_total ? a + rows.row(am) * a_pitch : nullptr;
    const uint8_t* brow = bc < columns ? b + size_t(bc) * k_bytes : nullptr;
    uint32_t acc[4][4] = {};  // unsigned byte dot products (u8 x u8)
    for (uint32_t k0 = 0; k0 < k_bytes; k0 += kTileK) {
        uint32_t kk = k0 + load_part * 16;
        uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
        if (arow && kk < k_bytes) va = *reinterpret_cast<const uint4*>(arow + kk);
        if (brow && kk < k_bytes) vb = *reinterpret_cast<const uint4*>(brow + kk);
        as[load_row][load_part * 4 + 0] = va.x;
        as[load_row][load_part * 4 + 1] = va.y;
        as[load_row][load_part * 4 + 2] = va.z;
        as[load_row][load_part * 4 + 3] = va.w;
        bs[load_row][load_part * 4 + 0] = vb.x;
        bs[load_row][load_part * 4 + 1] = vb.y;
        bs[load_row][load_part * 4 + 2] = vb.z;
        bs[load_row][load_part * 4 + 3] = vb.w;
        __syncthreads();
#pragma unroll
        for (int kw = 0; kw < kTileK / 4; ++kw) {
            uint32_t ra[4], rb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) ra[i] = as[tr * 4 + i][kw];
#pragma unroll
            for (int j = 0; j < 4; ++j) rb[j] = bs[tc * 4 + j][kw];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = __dp4a(ra[i], rb[j], acc[i][j]);
        }
        __syncthreads();
    }
    const uint32_t group = (c0 / 4) + tc;  // column group index (4 columns)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        uint32_t m = m0 + tr * 4 + i;
        if (m >= m_total) continue;
        if (epi.mode == kEpilogueRaw) {
            const uint64_t out_row = rows.row(m);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                uint32_t c = c0 + tc * 4 + j;
                if (c < columns) epi.raw[out_row * epi.raw_ld + c] = int32_t(acc[i][j]);
            }
            continue;
        }
        uint64_t s = uint64_t(uint32_t(acc[i][0])) + (uint64_t(uint32_t(acc[i][1])) << 8) +
                     (uint64_t(uint32_t(acc[i][2])) << 16) + (uint64_t(uint32_t(acc[i][3])) << 24);
        if (epi.mode == kEpilogueConvert) {
            if (group >= epi.r) continue;
            const DevicePrime f = epi.primes[group];
            uint32_t op, column;
            rows.residue(m, op, column);
            epi.residues[(size_t(op) * epi.r + group) * epi.n + column] = redc(s, f.p, f.pinv);
        } else {
            if (group < epi.words) epi.dots[rows.row(m) * epi.dots_stride + group] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// NTT: one CTA per length-N' transform, whole transform in shared memory.

__global__ void __launch_bounds__(512) ntt_forward_kernel(uint32_t* residues, const DevicePrime* __restrict__ primes,
                                                          const uint2* __restrict__ fwd, uint32_t r, uint32_t n,
                                                          uint32_t n_sub, uint32_t t_first, uint32_t op_first) {
    extern __shared__ uint32_t x[];
    const uint32_t t_index = t_first + blockIdx.x, k = blockIdx.y, op = op_first + blockIdx.z;
    const uint32_t p = primes[k].p;
    uint32_t* data = residues + (size_t(op) * r + k) * n + size_t(t_index) * n_sub;
    const uint2* table = fwd + size_t(k) * n_sub;
    for (uint32_t j = threadIdx.x; j < n_sub; j += blockDim.x) x[j] = data[j];
    __syncthreads();
    for (uint32_t m = 1, t = n_sub; m < n_sub; m *= 2) {
        t /= 2;
        for (uint32_t bfly = threadIdx.x; bfly < n_sub / 2; bfly += blockDim.x) {
            uint32_t i = bfly / t, jj = bfly - i * t, j = 2 * i * t + jj;
            uint2 w = table[m + i];
            uint32_t u = x[j], v = shoup(x[j + t], w.x, w.y, p);
            x[j] = add_mod(u, v, p);
            x[j + t] = sub_mod(u, v, p);
        }
        __syncthreads();
    }
    for (uint32_t j = threadIdx.x; j < n_sub; j += blockDim.x) data[j] = x[j];
}

__global__ void __launch_bounds__(512) ntt_inverse_kernel(uint32_t* residues, const DevicePrime* __restrict__ primes,
                                                          const uint2* __restrict__ inv, uint32_t r, uint32_t n,
                                                          uint32_t n_sub, uint32_t v_first) {
    extern __shared__ uint32_t x[];
    const uint32_t v_index = v_first + blockIdx.x, k = blockIdx.y;
    const DevicePrime f = primes[k];
    uint32_t* data = residues + size_t(k) * n + size_t(v_index) * n_sub;
    const uint2* table = inv + size_t(k) * n_sub;
    for (uint32_t j = threadIdx.x; j < n_sub; j += blockDim.x) x[j] = data[j];
    __syncthreads();
    for (uint32_t m = n_sub, t = 1; m > 1; m /= 2, t *= 2) {
        const uint32_t h = m / 2;
        for (uint32_t bfly = threadIdx.x; bfly < n_sub / 2; bfly += blockDim.x) {
            uint32_t i = bfly / t, jj = bfly - i * t, j = 2 * i * t + jj;
            uint2 w = table[h + i];
            uint32_t u = x[j], v = x[j + t];
            x[j] = add_mod(u, v, f.p);
            x[j + t] = shoup(sub_mod(u, v, f.p), w.x, w.y, f.p);
        }
        __syncthreads();
    }
    for (uint32_t j = threadIdx.x; j < n_sub; j += blockDim.x) data[j] = shoup(x[j], f.finish, f.finish_q, f.p);
}

// ---------------------------------------------------------------------------
// Register-blocked NTT for N' >= 256: 16 values per thread (N'/16 threads),
// up to four butterfly stages per pass between shared-memory exchanges.
// A pass of R stages on group g (2^R values spaced t_min apart, t_min = the
// smallest half-size in the pass) covers indices base + k*t_min, k < 2^R, with
// base = (g / t_min) * 2^R * t_min + g % t_min.

constexpr uint32_t kPerThread = 16;

// Shared-memory layout of a length-2^kLog transform: word i is stored at i ^ M(i >> 5), where M
// XORs column b into the bank bits when bit 5 + b of i is set. The columns were found by an
// exhaustive check of every warp access of every pass (forward and inverse, 16 values per
// thread): with them no pass has a bank conflict, where padding one word per 32 left 2-way
// conflicts in the passes with half-size 2 and 1 or 16. M is linear, and a pass's per-value
// offsets k t_min share no bits with its group base, so the swizzle of base + k t_min is the
// swizzle of base (once per group) XOR a compile-time constant.
template <uint32_t kLog>
__host__ __device__ constexpr uint32_t swizzle_column(int b) {
    constexpr uint32_t c8[] = {30, 1, 4};
    constexpr uint32_t c9[] = {7, 9, 27, 13};
    constexpr uint32_t c10[] = {27, 13, 8, 26, 8};
    constexpr uint32_t c11[] = {11, 1, 14, 20, 24, 27};
    constexpr uint32_t c12[] = {17, 26, 2, 21, 24, 25, 27};
    constexpr uint32_t c13[] = {7, 9, 27, 13, 8, 26, 8, 13};
    return kLog == 8 ? c8[b] : kLog == 9 ? c9[b] : kLog == 10 ? c10[b] : kLog == 11 ? c11[b] : kLog == 12 ? c12[b] : c13[b];
}

template <uint32_t kLog>
__host__ __device__ constexpr uint32_t swizzle(uint32_t i) {
    uint32_t m = 0;
    for (int b = 0; b < int(kLog) - 5; ++b)
        if ((i >> (5 + b)) & 1u) m ^= swizzle_column<kLog>(b);
    return i ^ m;
}

// Cooley-Tukey stages with half-sizes t_min*2^(R-1) .. t_min (forward, merged psi twiddles) on
// one group of 2^R values. With j = base + k*t_min and base = group_hi * 2^(log t_min + R) + off
// (off < t_min), butterfly (k, k + half) of stage r has twiddle m + (j >> (log t + 1))
// = m + group_hi * 2^r + (k >> (R - r)): the 2^(R-1-r) butterflies of block b = k >> (R - r)
// share one twiddle, so a pass loads 2^R - 1 twiddles for its R * 2^(R-1) butterflies.
// Values between stages are kept in [0, 2p) (2p < 2^32): each butterfly reduces its two inputs
// once, so that u + v and u - v + p stay below 2p, and multiplies by the twiddle without
// Shoup's final correction. Canonical inputs are a special case; the last pass reduces.
template <int R>
__device__ __forceinline__ void ct_stages(uint32_t (&x)[1 << R], uint32_t group_hi, uint32_t log_t_min,
                                          uint32_t log_n, const uint2* __restrict__ table, uint32_t p) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int half = 1 << (R - 1 - r);
        const uint32_t log_t = log_t_min + (R - 1 - r);  // this stage's half-size t = 2^log_t
        const uint32_t m = 1u << (log_n - 1 - log_t);     // number of groups: n / (2t)
#pragma unroll
        for (int b = 0; b < (1 << r); ++b) {
            const uint2 w = __ldg(&table[m + (group_hi << r) + b]);
#pragma unroll
            for (int k = b * 2 * half; k < b * 2 * half + half; ++k) {
                const uint32_t u = reduce_once(x[k], p);
                const uint32_t v = reduce_once(shoup_lazy(x[k + half], w.x, w.y, p), p);
                x[k] = u + v;
                x[k + half] = u - v + p;
            }
        }
    }
}

// Gentleman-Sande stages with half-sizes t_min .. t_min*2^(R-1) (inverse). Stage r's butterflies
// (k, k + 2^r) in block b = k >> (r + 1) share twiddle h + group_hi * 2^(R-1-r) + b.
// Values between stages are in [0, 2p), as in ct_stages.
template <int R>
__device__ __forceinline__ void gs_stages(uint32_t (&x)[1 << R], uint32_t group_hi, uint32_t log_t_min,
                                          uint32_t log_n, const uint2* __restrict__ table, uint32_t p) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int half = 1 << r;
        const uint32_t log_t = log_t_min + r;
        const uint32_t h = 1u << (log_n - 1 - log_t);
#pragma unroll
        for (int b = 0; b < (1 << (R - 1 - r)); ++b) {
            const uint2 w = __ldg(&table[h + (group_hi << (R - 1 - r)) + b]);
#pragma unroll
            for (int k = b * 2 * half; k < b * 2 * half + half; ++k) {
                const uint32_t u = reduce_once(x[k], p), v = reduce_once(x[k + half], p);
                x[k] = u + v;
                x[k + half] = shoup_lazy(u - v + p, w.x, w.y, p);
            }
        }
    }
}

// One pass of R stages over all of this thread's groups (transform length 2^kLog,
// 2^(kLog-4) threads). src/dst are shared (swizzled index) or global (plain index);
// kScale multiplies the values stored to global by (f, f_q).
template <int R, bool kForward, bool kFromGlobal, bool kToGlobal, bool kScale, uint32_t kLogTMin, uint32_t kLog>
__device__ __forceinline__ void ntt_pass(const uint32_t* src, uint32_t* dst, const uint2* __restrict__ table,
                                         uint32_t p, uint32_t f, uint32_t f_q) {
    constexpr int G = kPerThread >> R;  // groups per thread
    constexpr uint32_t kThreads = 1u << (kLog - 4);
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const uint32_t group = threadIdx.x + g * kThreads;
        const uint32_t off = group & ((1u << kLogTMin) - 1);
        const uint32_t base = ((group >> kLogTMin) << (kLogTMin + R)) + off;
        const uint32_t placed = swizzle<kLog>(base);  // shared-memory place of the group's first word
        // with t_min = 1 a group is 2^R consecutive words (base a multiple of 2^R): global
        // accesses go four words at a time (two in a one-stage pass), so a warp instruction
        // covers 16-byte (8-byte) pieces
        constexpr bool kVector = kLogTMin == 0 && R >= 2;
        constexpr bool kPair = kLogTMin == 0 && R == 1;
        uint32_t x[1 << R];
        if constexpr (kFromGlobal && kPair) {
            const uint2 w = *reinterpret_cast<const uint2*>(src + base);
            x[0] = w.x;
            x[1] = w.y;
        } else if constexpr (kFromGlobal && kVector) {
#pragma unroll
            for (int q = 0; q < (1 << R) / 4; ++q) {
                const uint4 w = reinterpret_cast<const uint4*>(src + base)[q];
                x[4 * q] = w.x;
                x[4 * q + 1] = w.y;
                x[4 * q + 2] = w.z;
                x[4 * q + 3] = w.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < (1 << R); ++k) {
                const uint32_t i = base + (uint32_t(k) << kLogTMin);
                x[k] = kFromGlobal ? src[i] : src[placed ^ swizzle<kLog>(uint32_t(k) << kLogTMin)];
            }
        }
        if (kForward)
            ct_stages<R>(x, group >> kLogTMin, kLogTMin, kLog, table, p);
        else
            gs_stages<R>(x, group >> kLogTMin, kLogTMin, kLog, table, p);
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
            if (kScale)
                x[k] = shoup(x[k], f, f_q, p);  // canonical: shoup takes any 32-bit value
            else if (kToGlobal)
                x[k] = reduce_once(x[k], p);    // [0, 2p) -> canonical
        }
        if constexpr (kToGlobal && kPair) {
            *reinterpret_cast<uint2*>(dst + base) = make_uint2(x[0], x[1]);
        } else if constexpr (kToGlobal && kVector) {
#pragma unroll
            for (int q = 0; q < (1 << R) / 4; ++q)
                reinterpret_cast<uint4*>(dst + base)[q] = make_uint4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
        } else {
#pragma unroll
            for (int k = 0; k < (1 << R); ++k) {
                const uint32_t i = base + (uint32_t(k) << kLogTMin);
                if (kToGlobal)
                    dst[i] = x[k];
                else
                    dst[placed ^ swizzle<kLog>(uint32_t(k) << kLogTMin)] = x[k];
            }
        }
    }
}

// Passes kDone.. of a length-2^kLog transform: four stages per pass, and a shorter pass for the
// remainder at the unit-stride end, where it touches global memory 2 consecutive words per
// thread instead of 16: last in the forward transform (half-sizes large -> small), first in the
// inverse (small -> large, which also scales its output).
template <bool kForward, uint32_t kLog, uint32_t kDone>
__device__ __forceinline__ void ntt_passes(uint32_t* data, uint32_t* xs, const uint2* __restrict__ table, uint32_t p,
                                           uint32_t f, uint32_t f_q) {
    constexpr int R = (!kForward && kDone == 0 && kLog % 4 != 0) ? int(kLog % 4)
                      : (kLog - kDone) < 4                       ? int(kLog - kDone)
                                                                  : 4;
    constexpr uint32_t kLogTMin = kForward ? kLog - kDone - R : kDone;
    constexpr bool kFirst = kDone == 0, kLast = kDone + R == kLog;
    ntt_pass<R, kForward, kFirst, kLast, kLast && !kForward, kLogTMin, kLog>(kFirst ? data : xs, kLast ? data : xs,
                                                                              table, p, f, f_q);
    if constexpr (!kLast) {
        __syncthreads();
        ntt_passes<kForward, kLog, kDone + R>(data, xs, table, p, f, f_q);
    }
}

// grid (op_count t_count, r): x = (op - op_first)*t_count + (t - t_first), y = prime, so a prime's
// transforms share its twiddles in L2
template <uint32_t kLog>
__global__ void __launch_bounds__(1u << (kLog - 4), (kLog >= 13 ? 2 : 4)) ntt_forward_blocked_kernel(
    uint32_t* residues, const DevicePrime* __restrict__ primes, const uint2* __restrict__ fwd, uint32_t r, uint32_t n,
    uint32_t t_first, uint32_t t_count, uint32_t op_first) {
    extern __shared__ uint32_t xs[];
    constexpr uint32_t kN = 1u << kLog;
    const uint32_t local_op = blockIdx.x / t_count, op = op_first + local_op;
    const uint32_t t_index = t_first + blockIdx.x - local_op * t_count, k = blockIdx.y;
    uint32_t* data = residues + (size_t(op) * r + k) * n + size_t(t_index) * kN;
    ntt_passes<true, kLog, 0>(data, xs, fwd + size_t(k) * kN, primes[k].p, 0, 0);
}

template <uint32_t kLog>
__global__ void __launch_bounds__(1u << (kLog - 4), (kLog >= 13 ? 2 : 4)) ntt_inverse_blocked_kernel(
    uint32_t* residues, const DevicePrime* __restrict__ primes, const uint2* __restrict__ inv, uint32_t r, uint32_t n,
    uint32_t v_first, uint32_t v_count, uint32_t /*op_first: the inverse works on operand row 0 only*/) {
    extern __shared__ uint32_t xs[];
    constexpr uint32_t kN = 1u << kLog;
    const uint32_t v_index = v_first + blockIdx.x, k = blockIdx.y;
    const DevicePrime f = primes[k];
    uint32_t* data = residues + size_t(k) * n + size_t(v_index) * kN;
    ntt_passes<false, kLog, 0>(data, xs, inv + size_t(k) * kN, f.p, f.finish, f.finish_q);
}

// C_v = sum_{t+u=v} A_t B_u + zeta * sum_{t+u=v+s} A_t B_u at every evaluation point,
// written over A_v. Products are Montgomery (x y 2^-32). Each thread takes V consecutive
// evaluation points (V = 2: 8-byte accesses, n_sub even).
template <int S, int V>
__global__ void pointwise_kernel(uint32_t* residues, const DevicePrime* __restrict__ primes,
                                 const uint2* __restrict__ zeta, uint32_t r, uint32_t n, uint32_t n_sub) {
    using Word = std::conditional_t<V == 2, uint2, uint32_t>;
    const uint32_t k = blockIdx.y;
    const uint32_t m = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    if (m >= n_sub) return;
    const DevicePrime f = primes[k];
    Word* a = reinterpret_cast<Word*>(residues + size_t(k) * n + m);
    const Word* b = reinterpret_cast<const Word*>(residues + (size_t(r) + k) * n + m);
    const size_t step = n_sub / V;  // one transform, in Words
    uint32_t av[V][S], bv[V][S];
#pragma unroll
    for (int t = 0; t < S; ++t) {
        const Word x = a[t * step], y = b[t * step];
        if constexpr (V == 2) {
            av[0][t] = x.x, av[1][t] = x.y, bv[0][t] = y.x, bv[1][t] = y.y;
        } else {
            av[0][t] = x, bv[0][t] = y;
        }
    }
    uint2 z[V];
    if constexpr (V == 2) {
        const uint4 zz = *reinterpret_cast<const uint4*>(zeta + size_t(k) * n_sub + m);
        z[0] = make_uint2(zz.x, zz.y), z[1] = make_uint2(zz.z, zz.w);
    } else {
        z[0] = zeta[size_t(k) * n_sub + m];
    }
    // two products per Montgomery reduction: a b + a' b' < 2 p^2 < p 2^32
#pragma unroll
    for (int v = 0; v < S; ++v) {
        uint32_t out[V];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            uint32_t low = 0, wrap = 0;
#pragma unroll
            for (int t = 0; t <= v; t += 2) {
                uint64_t pair = uint64_t(av[e][t]) * bv[e][v - t];
                if (t + 1 <= v) pair += uint64_t(av[e][t + 1]) * bv[e][v - t - 1];
                low = add_mod(low, redc(pair, f.p, f.pinv), f.p);
            }
#pragma unroll
            for (int t = v + 1; t < S; t += 2) {
                uint64_t pair = uint64_t(av[e][t]) * bv[e][v + S - t];
                if (t + 1 < S) pair += uint64_t(av[e][t + 1]) * bv[e][v + S - t - 1];
                wrap = add_mod(wrap, redc(pair, f.p, f.pinv), f.p);
            }
            out[e] = add_mod(low, shoup(wrap, z[e].x, z[e].y, f.p), f.p);
        }
        if constexpr (V == 2)
            a[v * step] = make_uint2(out[0], out[1]);
        else
            a[v * step] = out[0];
    }
}

// residues[0][k][v*N' + j] -> crt_in[s*j + v][k] (coefficient-major) for every transform v and
// j in [j_first, j_first + j_count), i.e. coefficients [s j_first, s (j_first + j_count)); zero for
// k in [r, r'). Block x covers up to 64 consecutive j of one transform and block y 64 primes, so
// every global access is a 256-byte run (two warp instructions of 128 bytes); the tile's rows are
// padded to 65 words, which keeps both the row-wise writes and the column-wise reads free of bank
// conflicts. 256 threads: 16 loads in flight per thread.
constexpr uint32_t kTransposeTile = 64;
__global__ void __launch_bounds__(256) transpose_kernel(const uint32_t* __restrict__ residues,
                                                        uint32_t* __restrict__ crt_in, uint32_t r, uint32_t padded_r,
                                                        uint32_t n, uint32_t log_split, uint32_t log_n_sub,
                                                        uint32_t j_first, uint32_t j_count) {
    __shared__ uint32_t tile[kTransposeTile][kTransposeTile + 1];
    const uint32_t blocks_per_v = (j_count + kTransposeTile - 1) / kTransposeTile, v = blockIdx.x / blocks_per_v;
    const uint32_t j0 = j_first + (blockIdx.x - v * blocks_per_v) * kTransposeTile, k0 = blockIdx.y * kTransposeTile;
    const uint32_t j_end = j_first + j_count, rho0 = (v << log_n_sub) + j0;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;  // 8 warps
#pragma unroll
    for (uint32_t row = warp; row < kTransposeTile; row += 8) {  // row = prime offset
        const uint32_t k = k0 + row;
#pragma unroll
        for (uint32_t half = 0; half < kTransposeTile; half += 32) {
            const uint32_t j = j0 + half + lane;
            tile[row][half + lane] = (k < r && j < j_end) ? residues[size_t(k) * n + rho0 + half + lane] : 0u;
        }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t row = warp; row < kTransposeTile; row += 8) {  // row = position offset
        const uint32_t j = j0 + row;
        if (j >= j_end) continue;
        uint32_t* out = crt_in + ((size_t(j) << log_split) + v) * padded_r;
#pragma unroll
        for (uint32_t half = 0; half < kTransposeTile; half += 32) {
            const uint32_t k = k0 + half + lane;
            if (k < padded_r) out[k] = tile[half + lane][row];
        }
    }
}

// ---------------------------------------------------------------------------
// Warp-wide multiword arithmetic over 32-word chunks.

// Carry into this lane given per-lane generate/propagate (mutually exclusive)
// and the chain bit entering lane 0; updates `chain` to the carry out of lane 31.
// Treats the 32 lanes as one 32-bit addition of (g|p) + g + chain.
__device__ __forceinline__ uint32_t chain_carry(bool generate, bool propagate, uint32_t& chain) {
    const uint32_t lane = threadIdx.x & 31;
    uint64_t g = __ballot_sync(kFull, generate), gp = g | __ballot_sync(kFull, propagate);
    uint64_t full = gp + g + chain;
    uint32_t carries = uint32_t(full ^ gp ^ g);
    chain = uint32_t(full >> 32);
    return (carries >> lane) & 1u;
}

__device__ __forceinline__ uint32_t word_or_zero(const uint32_t* v, int64_t at, uint32_t size) {
    return (at >= 0 && at < int64_t(size)) ? v[at] : 0u;
}

// bits [at, at+32) of the little-endian word array v (size words)
__device__ __forceinline__ uint32_t bits_word(const uint32_t* v, int64_t at, uint32_t size) {
    int64_t w = at >= 0 ? at / 32 : -((-at + 31) / 32);
    uint32_t offset = uint32_t(at - w * 32);
    uint64_t lo = word_or_zero(v, w, size), hi = word_or_zero(v, w + 1, size);
    return uint32_t(((hi << 32) | lo) >> offset);
}

// v[0..len) += term(w) (term < 2^32), with carry; returns the final carry.
template <class Term>
__device__ __forceinline__ uint32_t add_words(uint32_t* v, uint32_t len, Term term) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t chain = 0;
    for (uint32_t base = 0; base < len; base += 32) {
        uint32_t w = base + lane;
        uint32_t x = w < len ? v[w] : 0u, y = w < len ? term(w) : 0u;
        uint64_t sum = uint64_t(x) + y;
        uint32_t low = uint32_t(sum);
        uint32_t carry = chain_carry((sum >> 32) != 0, low == kFull, chain);
        if (w < len) v[w] = low + carry;
    }
    __syncwarp();
    return chain;
}

// v[0..len) -= term(w), with borrow; returns the final borrow.
template <class Term>
__device__ __forceinline__ uint32_t sub_words(uint32_t* v, uint32_t len, Term term) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t chain = 0;
    for (uint32_t base = 0; base < len; base += 32) {
        uint32_t w = base + lane;
        uint32_t x = w < len ? v[w] : 0u, y = w < len ? term(w) : 0u;
        uint32_t borrow = chain_carry(x < y, x == y, chain);
        if (w < len) v[w] = x - y - borrow;
    }
    __syncwarp();
    return chain;
}

// sign of (v - q) over len words (q[w] = 0 for w >= limbs): -1, 0, 1
__device__ __forceinline__ int compare_q(const uint32_t* v, uint32_t len, const uint32_t* q, uint32_t limbs) {
    const uint32_t lane = threadIdx.x & 31;
    for (int64_t base = int64_t((len + 31) / 32 - 1) * 32; base >= 0; base -= 32) {
        uint32_t w = uint32_t(base) + lane;
        uint32_t x = w < len ? v[w] : 0u, y = w < limbs ? q[w] : 0u;
        uint32_t differ = __ballot_sync(kFull, x != y);
        if (differ) {
            uint32_t top = 31 - __clz(differ);
            int less = __shfl_sync(kFull, x < y ? 1 : 0, top);
            return less ? -1 : 1;
        }
    }
    return 0;
}

// One warp per coefficient; its words live in shared memory.
//
// The CRT word sums split cleanly: words [0, L+2) are a carry-save form of
// T = sum v_k M_k (< 2^(32(L+2)), so nothing carries out of them), words
// L+2..L+4 a carry-save form of D = sum v_k floor(2^64/p_k). Hence
//   K  = (D + 2^63) >> 64 straight from three word sums,
//   T' = T + K*(-P mod q) in one carry pass over dots[w] + K*R[w],
//   c  = T' - quotient*q in one signed carry pass, then at most three q's off.
__global__ void reduce_kernel(ReduceParams prm, uint32_t stride) {
    extern __shared__ uint32_t scratch[];
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x & 31;
    const uint32_t warps = blockDim.x / 32;
    uint32_t* v = scratch + size_t(warp) * stride;
    const uint32_t limbs = prm.limbs, tlen = limbs + 2;
    const uint32_t* q = prm.q;
    for (uint32_t i = blockIdx.x * warps + warp; i < prm.n; i += gridDim.x * warps) {
        const uint64_t* d = prm.dots + size_t(i) * prm.dots_stride;
        // 1. K = (D + 2^63) >> 64, D = d[L+2] + d[L+3] 2^32 + d[L+4] 2^64 (each word sum < 2^56)
        const uint64_t x0 = d[limbs + 2], x1 = d[limbs + 3], x2 = d[limbs + 4];
        const uint64_t low = x0 + (x1 << 32);
        const uint64_t high = (x1 >> 32) + x2 + (low < x0 ? 1 : 0);  // D = high 2^64 + low
        const uint64_t kq = high + ((low + (1ull << 63)) < low ? 1 : 0);
        // 2. T' = sum_w (d[w] + K R[w]) 2^(32w), collapsed to exact words in one carry pass. A lane
        //    holds words w0 = base + 2 lane and w0 + 1 of a 64-word step: its two word sums meet
        //    in-lane, the bits at 2^64 and up go to the next lane by a shuffle (< 2^25), and one
        //    warp-wide carry resolution covers 64 words. The word sums come from DRAM in 16-byte
        //    pairs, kBatch steps' worth before any is used, so one load latency covers kBatch steps
        //    of the (serial) carry chain. K < 2r fits 32 bits.
        constexpr uint32_t kBatch = 4;
        const uint32_t k32 = uint32_t(kq);
        uint32_t chain = 0, carried_high = 0;
        for (uint32_t batch = 0; batch < tlen; batch += 64 * kBatch) {
            uint64_t x0[kBatch], x1[kBatch];
#pragma unroll
            for (uint32_t u = 0; u < kBatch; ++u) {
                const uint32_t w0 = batch + 64 * u + 2 * lane;
                uint64_t d0 = 0, d1 = 0;
                if (w0 < tlen) {  // w0 + 1 < dots_stride: the row holds at least tlen + 3 words
                    const ulonglong2 pair = *reinterpret_cast<const ulonglong2*>(d + w0);
                    d0 = pair.x;
                    d1 = w0 + 1 < tlen ? pair.y : 0ull;
                }
                const uint32_t r0 = w0 < limbs ? prm.minus_p[w0] : 0u, r1 = w0 + 1 < limbs ? prm.minus_p[w0 + 1] : 0u;
                x0[u] = d0 + uint64_t(k32) * r0;  // < 2^57
                x1[u] = d1 + uint64_t(k32) * r1;
            }
#pragma unroll
            for (uint32_t u = 0; u < kBatch; ++u) {
                const uint32_t base = batch + 64 * u;
                if (base >= tlen) break;  // warp-uniform
                const uint32_t w0 = base + 2 * lane;
                const uint32_t top = uint32_t(x1[u] >> 32);
                uint32_t below = __shfl_up_sync(kFull, top, 1);
                if (lane == 0) below = carried_high;
                carried_high = __shfl_sync(kFull, top, 31);
                const uint64_t s0 = uint64_t(uint32_t(x0[u])) + below;                     // < 2^33
                const uint64_t s1 = (x0[u] >> 32) + uint32_t(x1[u]) + uint32_t(s0 >> 32);  // < 2^33
                uint32_t word0 = uint32_t(s0), word1 = uint32_t(s1);
                const bool generate = (s1 >> 32) != 0;
                const uint32_t carry = chain_carry(generate, !generate && (word0 & word1) == kFull, chain);
                word0 += carry;
                word1 += (carry != 0 && word0 == 0) ? 1u : 0u;
                if (w0 < tlen) v[w0] = word0;
                if (w0 + 1 < tlen) v[w0 + 1] = word1;
            }
        }
        __syncwarp();
        // 3. Barrett quotient from the 128 bits of T' at q's top-64-bit window
        const uint64_t tl = uint64_t(bits_word(v, prm.top_shift, tlen)) |
                            (uint64_t(bits_word(v, int64_t(prm.top_shift) + 32, tlen)) << 32);
        const uint64_t th = uint64_t(bits_word(v, int64_t(prm.top_shift) + 64, tlen)) |
                            (uint64_t(bits_word(v, int64_t(prm.top_shift) + 96, tlen)) << 32);
        const uint64_t prod_l_hi = __umul64hi(tl, prm.mu_low);
        const uint64_t prod_h_lo = th * prm.mu_low, prod_h_hi = __umul64hi(th, prm.mu_low);
        const uint64_t word1 = prod_l_hi + prod_h_lo;
        const uint64_t word2 = prod_h_hi + (word1 < prod_l_hi ? 1 : 0);
        const uint64_t quotient = th + word2 + ((tl + word1 < tl) ? 1 : 0);
        const uint32_t ql = uint32_t(quotient), qh = uint32_t(quotient >> 32);
        __syncwarp();
        // 4. c = T' - quotient*q in one signed carry pass, two words per lane as in step 2. With
        //    a_w = ql q[w], b_w = qh q[w-1]:
        //    z_w = T'[w] - lo(a_w) - lo(b_w) - hi(a_{w-1}) - hi(b_{w-1})  in (-2^35, 2^32),
        //    c_w = floor(z_w / 2^32) in [-8, 0] moves to word w + 1, leaving sw_w in [-8, 2^32) and a
        //    one-bit borrow chain. A lane generates a borrow when sw1 < 0, or sw1 = 0 and sw0 < 0,
        //    and passes one on when sw1 = sw0 = 0.
        chain = 0;
        uint64_t carry_hi = 0;  // hi(a)+hi(b) of the previous step's last word
        int32_t carry_c = 0;    // signed word carry of the previous step's last word
        for (uint32_t base = 0; base < tlen; base += 64) {
            const uint32_t w0 = base + 2 * lane, w1 = w0 + 1;
            const uint32_t qa = w0 < limbs ? q[w0] : 0u, qb = w1 < limbs ? q[w1] : 0u;
            const uint32_t qm = (w0 >= 1 && w0 - 1 < limbs) ? q[w0 - 1] : 0u;
            const uint64_t a0 = uint64_t(ql) * qa, b0 = uint64_t(qh) * qm;  // word w0
            const uint64_t a1 = uint64_t(ql) * qb, b1 = uint64_t(qh) * qa;  // word w1
            const uint64_t hi0 = (a0 >> 32) + (b0 >> 32), hi1 = (a1 >> 32) + (b1 >> 32);
            uint64_t hi_below = (uint64_t(__shfl_up_sync(kFull, uint32_t(hi1 >> 32), 1)) << 32) |
                                __shfl_up_sync(kFull, uint32_t(hi1), 1);
            if (lane == 0) hi_below = carry_hi;
            carry_hi = (uint64_t(__shfl_sync(kFull, uint32_t(hi1 >> 32), 31)) << 32) | __shfl_sync(kFull, uint32_t(hi1), 31);
            const uint64_t e0 = (a0 & 0xffffffffull) + (b0 & 0xffffffffull) + hi_below;
            const uint64_t e1 = (a1 & 0xffffffffull) + (b1 & 0xffffffffull) + hi0;
            const int64_t z0 = int64_t(w0 < tlen ? v[w0] : 0u) - int64_t(e0);
            const int64_t z1 = int64_t(w1 < tlen ? v[w1] : 0u) - int64_t(e1);
            const int32_t c0 = int32_t(z0 >> 32), c1 = int32_t(z1 >> 32);
            int32_t c_below = __shfl_up_sync(kFull, c1, 1);
            if (lane == 0) c_below = carry_c;
            carry_c = __shfl_sync(kFull, c1, 31);
            const int64_t sw0 = int64_t(uint32_t(z0)) + c_below, sw1 = int64_t(uint32_t(z1)) + c0;
            const bool generate = sw1 < 0 || (sw1 == 0 && sw0 < 0);
            const uint32_t borrow = chain_carry(generate, !generate && sw1 == 0 && sw0 == 0, chain);
            const int64_t t0 = sw0 - borrow;
            if (w0 < tlen) v[w0] = uint32_t(t0);
            if (w1 < tlen) v[w1] = uint32_t(sw1 - (t0 < 0 ? 1 : 0));
        }
        __syncwarp();
        // 5. at most three subtractions of q remain
        int corrections = 0;
        while (compare_q(v, tlen, q, limbs) >= 0) {
            if (++corrections > 3) {
                if (lane == 0) atomicOr(prm.error_flag, 1u);
                break;
            }
            sub_words(v, tlen, [&](uint32_t w) { return w < limbs ? q[w] : 0u; });
        }
        // 6. canonical result
        uint32_t* out = prm.out + size_t(i) * limbs;
        for (uint32_t w = lane; w < limbs; w += 32) out[w] = v[w];
        __syncwarp();
    }
}


uint32_t log2_u32(uint32_t x) { return x ? 31 - __builtin_clz(x) : 0; }

}  // namespace

void launch_pad_operands(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n, uint32_t limbs,
                         uint32_t padded_limbs, uint32_t split, cudaStream_t stream) {
    const uint32_t log_split = log2_u32(split), log_n_sub = log2_u32(n) - log_split;
    const uint32_t blocks = std::min<uint32_t>((2 * n + 7) / 8, 148 * 16);  // 8 rows (warps) per block
    pad_operands_kernel<<<blocks, 256, 0, stream>>>(a, b, out, n, limbs, padded_limbs, log_split, log_n_sub);
}

void launch_pad_rows(const uint32_t* staged, uint32_t* out, uint32_t n, uint32_t limbs, uint32_t padded_limbs,
                     uint32_t split, uint32_t first_row, uint32_t count, cudaStream_t stream, uint32_t op_first,
                     uint32_t op_count) {
    const uint32_t log_split = log2_u32(split), log_n_sub = log2_u32(n) - log_split;
    const uint32_t blocks = std::min<uint32_t>((op_count * count + 7) / 8, 148 * 16);
    pad_rows_kernel<<<blocks, 256, 0, stream>>>(staged, out, n, limbs, padded_limbs, log_split, log_n_sub, first_row,
                                                count, op_first, op_count);
}

void launch_twiddles(const DevicePrime* primes, uint32_t r, uint32_t n_sub, uint2* fwd, uint2* inv, uint2* zeta,
                     cudaStream_t stream) {
    dim3 grid((n_sub + 255) / 256, r);
    twiddles_kernel<<<grid, 256, 0, stream>>>(primes, r, n_sub, log2_u32(n_sub), fwd, inv, zeta);
}

void launch_convert_weights(const DevicePrime* primes, uint32_t r, uint32_t padded_r, uint32_t limbs,
                            uint32_t k_bytes, uint8_t* out, cudaStream_t stream) {
    dim3 grid((k_bytes + 255) / 256, padded_r);
    convert_weights_kernel<<<grid, 256, 0, stream>>>(primes, r, padded_r, limbs, k_bytes, out);
}

void launch_crt_weights(const uint32_t* weights_words, uint32_t r, uint32_t padded_r, uint32_t words,
                        uint32_t columns, uint8_t* out, cudaStream_t stream) {
    dim3 grid((4 * padded_r + 255) / 256, columns);
    crt_weights_kernel<<<grid, 256, 0, stream>>>(weights_words, r, padded_r, words, columns, out);
}

void launch_gemm_simt(const uint8_t* a, uint64_t a_pitch, RowMap rows, uint32_t m, const uint8_t* b,
                      uint32_t columns, uint32_t k_bytes, const Epilogue& epilogue, cudaStream_t stream) {
    dim3 grid((m + kTile - 1) / kTile, (columns + kTile - 1) / kTile);
    gemm_simt_kernel<<<grid, 256, 0, stream>>>(a, a_pitch, rows, m, b, columns, k_bytes, epilogue);
}

static uint32_t ntt_threads(uint32_t n_sub) {
    uint32_t half = n_sub / 2;
    return half >= 512 ? 512 : (half >= 32 ? half : 32);
}

template <bool kForward, uint32_t kLog>
static void launch_blocked(uint32_t* residues, const DevicePrime* primes, const uint2* table, uint32_t r, uint32_t n,
                           uint32_t first, uint32_t count, cudaStream_t stream, uint32_t op_first, uint32_t op_count) {
    constexpr uint32_t kN = 1u << kLog;
    const size_t smem = kN * sizeof(uint32_t);
    auto kernel = kForward ? ntt_forward_blocked_kernel<kLog> : ntt_inverse_blocked_kernel<kLog>;
    static bool configured = false;
    if (!configured) {  // room for several transforms per SM
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        configured = true;
    }
    dim3 grid(kForward ? op_count * count : count, r);
    kernel<<<grid, kN / kPerThread, smem, stream>>>(residues, primes, table, r, n, first, count, op_first);
}

template <bool kForward>
static bool launch_blocked_any(uint32_t n_sub, uint32_t* residues, const DevicePrime* primes, const uint2* table,
                               uint32_t r, uint32_t n, uint32_t first, uint32_t count, cudaStream_t stream,
                               uint32_t op_first = 0, uint32_t op_count = 2) {
#define NEGACYCLIC_BLOCKED(LOG) \
    launch_blocked<kForward, LOG>(residues, primes, table, r, n, first, count, stream, op_first, op_count)
    switch (n_sub) {
        case 256: NEGACYCLIC_BLOCKED(8); return true;
        case 512: NEGACYCLIC_BLOCKED(9); return true;
        case 1024: NEGACYCLIC_BLOCKED(10); return true;
        case 2048: NEGACYCLIC_BLOCKED(11); return true;
        case 4096: NEGACYCLIC_BLOCKED(12); return true;
        case 8192: NEGACYCLIC_BLOCKED(13); return true;
        default: return false;
    }
#undef NEGACYCLIC_BLOCKED
}

void launch_ntt_forward(uint32_t* residues, const DevicePrime* primes, const uint2* fwd, uint32_t r, uint32_t n,
                        uint32_t n_sub, uint32_t t_first, uint32_t t_count, cudaStream_t stream, uint32_t op_first,
                        uint32_t op_count) {
    if (launch_blocked_any<true>(n_sub, residues, primes, fwd, r, n, t_first, t_count, stream, op_first, op_count))
        return;
    dim3 grid(t_count, r, op_count);
    ntt_forward_kernel<<<grid, ntt_threads(n_sub), n_sub * sizeof(uint32_t), stream>>>(residues, primes, fwd, r, n,
                                                                                          n_sub, t_first, op_first);
}

void launch_ntt_inverse(uint32_t* residues, const DevicePrime* primes, const uint2* inv, uint32_t r, uint32_t n,
                        uint32_t n_sub, uint32_t v_first, uint32_t v_count, cudaStream_t stream) {
    if (launch_blocked_any<false>(n_sub, residues, primes, inv, r, n, v_first, v_count, stream)) return;
    dim3 grid(v_count, r);
    ntt_inverse_kernel<<<grid, ntt_threads(n_sub), n_sub * sizeof(uint32_t), stream>>>(residues, primes, inv, r, n,
                                                                                          n_sub, v_first);
}

void launch_pointwise(uint32_t* residues, const DevicePrime* primes, const uint2* zeta, uint32_t r, uint32_t n,
                      uint32_t n_sub, uint32_t split, cudaStream_t stream) {
    if (n_sub % 2 == 0) {  // two evaluation points per thread
        dim3 grid((n_sub / 2 + 127) / 128, r);
        switch (split) {
            case 1: pointwise_kernel<1, 2><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
            case 2: pointwise_kernel<2, 2><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
            case 4: pointwise_kernel<4, 2><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
            case 8: pointwise_kernel<8, 2><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
            default: pointwise_kernel<16, 2><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
        }
        return;
    }
    dim3 grid((n_sub + 127) / 128, r);
    switch (split) {
        case 1: pointwise_kernel<1, 1><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
        case 2: pointwise_kernel<2, 1><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
        case 4: pointwise_kernel<4, 1><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
        case 8: pointwise_kernel<8, 1><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
        default: pointwise_kernel<16, 1><<<grid, 128, 0, stream>>>(residues, primes, zeta, r, n, n_sub); break;
    }
}

void launch_transpose(const uint32_t* residues, uint32_t* crt_in, uint32_t r, uint32_t padded_r, uint32_t n,
                      uint32_t split, uint32_t j_first, uint32_t j_count, cudaStream_t stream) {
    const uint32_t log_split = log2_u32(split), log_n_sub = log2_u32(n) - log_split;
    dim3 grid(split * ((j_count + kTransposeTile - 1) / kTransposeTile), (padded_r + kTransposeTile - 1) / kTransposeTile);
    transpose_kernel<<<grid, 256, 0, stream>>>(residues, crt_in, r, padded_r, n, log_split, log_n_sub, j_first,
                                               j_count);
}

void launch_reduce(const ReduceParams& params, cudaStream_t stream) {
    const uint32_t stride = (params.words + 1 + 31) / 32 * 32;
    // up to 8 warps (coefficients) per block, each with `stride` words of shared memory
    constexpr size_t kSmemBudget = 200 * 1024;
    uint32_t warps = uint32_t(std::min<size_t>(8, std::max<size_t>(1, kSmemBudget / (stride * sizeof(uint32_t)))));
    const size_t smem = size_t(warps) * stride * sizeof(uint32_t);
    if (smem > 48 * 1024)  // per device; cheap enough to repeat
        cudaFuncSetAttribute(reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBudget));
    uint32_t blocks = (params.n + warps - 1) / warps;
    if (blocks > 148u * 8) blocks = 148u * 8;
    reduce_kernel<<<blocks, warps * 32, smem, stream>>>(params, stride);
}

}  // namespace negacyclic
