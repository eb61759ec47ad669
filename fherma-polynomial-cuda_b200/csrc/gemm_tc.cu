// tcgen05 kind::i8 GEMM with TMA loads, an mbarrier pipeline and TMEM accumulators.
//
// Replaces the reference's sm_80 warp-MMA byte GEMM (tensor_product,
// src/solve.cu:88-142: mma.sync m16n8k32 u8.u8.s32 with 64x16-word tiles) with
// the Blackwell path: one CTA computes a 128 x 256 tile of D = A B^T
// (A: [M][K] u8, B: [N][K] u8, both K-major), one thread issues
// tcgen05.mma.cta_group::1.kind::i8 (M=128, N=256, K=32 bytes per instruction)
// from 128B-swizzled shared-memory tiles that TMA fills through a 4-stage ring,
// the s32 accumulator lives in 256 TMEM columns, and the epilogue reads it back
// with tcgen05.ld and applies the conversion (REDC) or CRT (word sum) step.
//
// Exactness: each accumulator is a sum of K products of bytes, K * 255^2 < 2^31
// for K <= 33024 (checked by the plan), so s32 accumulation is exact.
//
// Persistent (one CTA per SM) and warp-specialised: warp 0 = TMA producer,
// warp 1 = MMA issuer and TMEM owner (two 256-column accumulators), warps 2-5 =
// epilogue, so the epilogue of one tile overlaps the MMAs of the next. Every
// mbarrier wait is bounded (TileShape::limit cycles of SM clock, ~2 s by
// default) and also ends when another role raised the abort flag. On a timeout
// the kernel records an error bit (in the caller's status word and in a
// device-wide word), raises the flag (in both CTAs of a pair), lets the
// copies it issued land, frees TMEM and returns.
#include <cuda.h>

#include <cstdio>
#include <cstdlib>

#include "gemm_tc.cuh"

namespace negacyclic {

namespace {

constexpr uint32_t kBlockM = 128, kBlockN = 256, kBlockK = 128;  // K in bytes (one 128B swizzle atom)
constexpr uint32_t kStages = 4;
constexpr uint32_t kATileBytes = kBlockM * kBlockK;                // 16 KB
constexpr uint32_t kBTileBytes = kBlockN * kBlockK;                // 32 KB
constexpr uint32_t kStageBytes = kATileBytes + kBTileBytes;
constexpr uint32_t kAccColumns = 256;                            // one 128 x 256 s32 accumulator
constexpr uint32_t kEpilogueWarps = 4;
constexpr uint32_t kThreads = 64 + 32 * kEpilogueWarps;
constexpr long long kDefaultLimitCycles = 4000000000ll;  // ~2 s at 1.9 GHz
constexpr uint64_t kAbortDrainNs = 1000000;               // 1 ms: in-flight TMA loads land long before
constexpr size_t kSmemBytes = size_t(kStages) * kStageBytes + 1024 /*align*/ + 256 /*barriers, TMEM slot*/;

__device__ uint32_t g_tc_error;
__device__ uint32_t g_tile_counter;  // tile counter of GEMMs without one of their own

// Instruction descriptor: D s32, A/B unsigned 8-bit, both K-major, M=128, N=256.
constexpr uint32_t kInstrDesc = (2u << 4)              /* c_format = S32 */
                                | (0u << 7) | (0u << 10) /* a/b format = u8 */
                                | (0u << 15) | (0u << 16) /* K-major */
                                | ((kBlockN >> 3) << 17) | ((kBlockM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(ptr));
}

// UMMA shared-memory descriptor for a K-major tile in the canonical 128B-swizzle
// layout: rows of 128 bytes, 8-row core groups 1024 bytes apart (SBO), tile base
// 1024-byte aligned (base offset 0), descriptor version 1.
__device__ __forceinline__ uint64_t smem_descriptor(uint32_t addr) {
    uint64_t d = 0;
    d |= uint64_t((addr & 0x3FFFFu) >> 4);
    d |= uint64_t(1) << 16;           // leading byte offset (unused for swizzled K-major)
    d |= uint64_t(1024 >> 4) << 32;   // stride byte offset
    d |= uint64_t(1) << 46;           // version
    d |= uint64_t(2) << 61;           // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity to complete: false after `limit` cycles, or
// (when `abort` is given) as soon as another role has raised the abort flag.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit,
                                          const volatile uint32_t* abort = nullptr) {
    const long long start = clock64();
    for (uint32_t i = 0;; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 63u) == 63u && ((abort && *abort) || clock64() - start > limit)) return false;
    }
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// After an abort: keep the CTA (and, through the final cluster barrier, its peer) resident for
// kAbortDrainNs, so that TMA loads still in flight land in live shared memory. The wait is
// bounded by %globaltimer; a TMA load completes within microseconds.
__device__ __forceinline__ void abort_drain() {
    const uint64_t start = global_ns();
    while (global_ns() - start < kAbortDrainNs) {
    }
}

// Records a pipeline error: the device-wide diagnostic word and, when given, the caller's status
// word (bits shifted into NEGACYCLIC_STATUS_GEMM_MASK).
__device__ __forceinline__ void record_error(uint32_t* status, uint32_t bit) {
    atomicOr(&g_tc_error, bit);
    if (status) atomicOr(status, bit << 8);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t desc_a, uint64_t desc_b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(desc_a), "l"(desc_b), "r"(kInstrDesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_load32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct TileShape {
    uint32_t m, columns, k_tiles, m_tiles, n_tiles, group_m;
    RowMap rows;
    uint32_t* tile_counter;  // pair kernel: next unclaimed tile (zero at launch)
    uint32_t* status;        // caller's status word (NEGACYCLIC_STATUS_*), or nullptr
    long long limit;         // cycles any one pipeline wait may take
    uint32_t withheld;       // diagnostics: CTA (pair) 0's producer stops before this pipeline step
};

// Tile index -> (m tile, n tile) in groups of group_m m-tiles, m fastest, so the
// CTAs running at the same time share B tiles (and their A tiles stay in L2).
__device__ __forceinline__ void tile_coords(uint32_t tile, const TileShape& shape, uint32_t& m_tile,
                                            uint32_t& n_tile) {
    const uint32_t span = shape.group_m * shape.n_tiles;
    const uint32_t group = tile / span, within = tile - group * span;
    const uint32_t first_m = group * shape.group_m;
    const uint32_t rows_in_group = min(shape.group_m, shape.m_tiles - first_m);
    m_tile = first_m + within % rows_in_group;
    n_tile = within / rows_in_group;
}

// Applies the epilogue to 32 accumulator columns (c_base .. c_base+31) of one row.
// Raw and CRT epilogues of one 32-column chunk of a row (lane = row).
__device__ __forceinline__ void epilogue_chunk(const Epilogue& epi, const uint32_t (&v)[32], uint32_t c_base,
                                               uint32_t columns, uint64_t out_row) {
    if (epi.mode == kEpilogueRaw) {
        int32_t* out = epi.raw + out_row * epi.raw_ld;
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (c_base + j < columns) out[c_base + j] = int32_t(v[j]);
        return;
    }
    uint64_t sum[8];
#pragma unroll
    for (int g = 0; g < 8; ++g)
        sum[g] = uint64_t(v[4 * g]) + (uint64_t(v[4 * g + 1]) << 8) + (uint64_t(v[4 * g + 2]) << 16) +
                 (uint64_t(v[4 * g + 3]) << 24);
    // the lane's 8 words are consecutive in its row: two whole 32-byte sectors (the work space is
    // 256-byte aligned, rows are a multiple of 8 words, the chunk starts at a multiple of 8 words)
    const uint32_t g0 = c_base / 4;
    if (g0 >= epi.words) return;
    uint64_t* out = epi.dots + out_row * epi.dots_stride + g0;
    if (g0 + 8 <= epi.dots_stride && (epi.dots_stride & 3) == 0) {
        asm volatile("st.global.v4.b64 [%0], {%1, %2, %3, %4};" ::"l"(out), "l"(sum[0]), "l"(sum[1]), "l"(sum[2]),
                     "l"(sum[3])
                     : "memory");
        asm volatile("st.global.v4.b64 [%0], {%1, %2, %3, %4};" ::"l"(out + 4), "l"(sum[4]), "l"(sum[5]),
                     "l"(sum[6]), "l"(sum[7])
                     : "memory");
        return;
    }
#pragma unroll
    for (int g = 0; g < 8; ++g)
        if (g0 + g < epi.words) out[g] = sum[g];
}

// One epilogue warp's share of an accumulator: 32 rows (one per lane) x 256 columns starting at
// col0, read from TMEM at t_base in 32-column chunks.
// Conversion: column group g = 4k..4k+3 holds the byte dots of prime k; the residue is
// REDC(sum_d G_d 256^d). The tile's 64 primes are loaded once (lane l: groups l and l + 32)
// and broadcast by shuffles, instead of one dependent table load per group.
__device__ __forceinline__ void epilogue_rows(const Epilogue& epi, uint32_t t_base, uint32_t col0, uint32_t columns,
                                              bool row_ok, uint64_t out_row, uint32_t op, uint32_t column,
                                              uint32_t lane) {
    if (epi.mode == kEpilogueConvert) {
        const uint32_t g0 = col0 / 4;
        uint32_t p_lo = 1, pinv_lo = 0, p_hi = 1, pinv_hi = 0;
        if (g0 + lane < epi.r) {
            p_lo = epi.primes[g0 + lane].p;
            pinv_lo = epi.primes[g0 + lane].pinv;
        }
        if (g0 + 32 + lane < epi.r) {
            p_hi = epi.primes[g0 + 32 + lane].p;
            pinv_hi = epi.primes[g0 + 32 + lane].pinv;
        }
        uint32_t* out = epi.residues + size_t(op) * epi.r * epi.n + column;  // + k * N for prime k
        for (uint32_t chunk = 0; chunk < kBlockN / 32; ++chunk) {
            const uint32_t c_base = col0 + chunk * 32;
            if (c_base >= columns) break;  // warp-uniform
            uint32_t v[32];
            tmem_load32(t_base + chunk * 32, v);
            const uint32_t from_p = chunk < 4 ? p_lo : p_hi, from_pinv = chunk < 4 ? pinv_lo : pinv_hi;
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                const uint32_t source = (chunk & 3) * 8 + g, k = c_base / 4 + g;
                const uint32_t p = __shfl_sync(0xffffffffu, from_p, source);
                const uint32_t pinv = __shfl_sync(0xffffffffu, from_pinv, source);
                const uint64_t s = uint64_t(v[4 * g]) + (uint64_t(v[4 * g + 1]) << 8) +
                                   (uint64_t(v[4 * g + 2]) << 16) + (uint64_t(v[4 * g + 3]) << 24);
                if (row_ok && k < epi.r) out[size_t(k) * epi.n] = redc(s, p, pinv);
            }
        }
        return;
    }
    for (uint32_t chunk = 0; chunk < kBlockN / 32; ++chunk) {
        const uint32_t c_base = col0 + chunk * 32;
        if (c_base >= columns) break;  // warp-uniform
        uint32_t v[32];
        tmem_load32(t_base + chunk * 32, v);
        if (row_ok) epilogue_chunk(epi, v, c_base, columns, out_row);
    }
}

// Persistent, warp-specialised GEMM: each CTA walks tiles blockIdx.x, +gridDim.x, ...
//   warp 0 (one thread)  TMA producer over a kStages-deep shared-memory ring
//   warp 1 (one thread)  MMA issuer; the whole warp allocates / frees 512 TMEM columns
//   warps 2-5            epilogue; two 256-column accumulators alternate between tiles,
//                        so tile i's epilogue overlaps tile i+1's MMAs
__global__ void __launch_bounds__(kThreads, 1) gemm_tc_kernel(const __grid_constant__ CUtensorMap a_map,
                                                              const __grid_constant__ CUtensorMap b_map,
                                                              TileShape shape, Epilogue epi) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* a_smem = smem;
    uint8_t* b_smem = smem + kStages * kATileBytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(b_smem + kStages * kBTileBytes);
    uint64_t* empty = full + kStages;
    uint64_t* acc_full = empty + kStages;  // [2] MMA -> epilogue
    uint64_t* acc_empty = acc_full + 2;    // [2] epilogue -> MMA
    uint64_t* drain = acc_empty + 2;       // MMA warp's final completion
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile uint32_t* abort_flag = tmem_slot + 1;

    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t tiles = shape.m_tiles * shape.n_tiles;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (uint32_t a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], kEpilogueWarps);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * kAccColumns)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer
            uint32_t step = 0, issued = 0;
            bool ok = true, withheld = false;
            for (uint32_t tile = blockIdx.x; tile < tiles && ok && !withheld; tile += gridDim.x) {
                uint32_t m_tile, n_tile;
                tile_coords(tile, shape, m_tile, n_tile);
                const uint32_t row0 = m_tile * kBlockM, col0 = n_tile * kBlockN;
                // operand row of the tile's first row; its 128 rows are consecutive in memory
                const uint32_t a_row = uint32_t(shape.rows.row(row0));
                for (uint32_t ks = 0; ks < shape.k_tiles; ++ks, ++step) {
                    const uint32_t s = step % kStages, round = step / kStages;
                    if (blockIdx.x == 0 && step == shape.withheld) {  // diagnostics: a stage that never comes
                        withheld = true;
                        break;
                    }
                    if (*abort_flag || !mbar_wait(&empty[s], (round & 1) ^ 1, shape.limit, abort_flag)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full[s], kStageBytes);
                    tma_load_2d(a_smem + s * kATileBytes, &a_map, &full[s], int(ks * kBlockK), int(a_row));
                    tma_load_2d(b_smem + s * kBTileBytes, &b_map, &full[s], int(ks * kBlockK), int(col0));
                    issued = step + 1;
                }
            }
            if (!ok) {
                *abort_flag = 1;
                record_error(shape.status, 1u);
                // let the loads already issued land before the CTA can exit (each of these phases
                // completes: this thread armed it and issued all of its bytes)
                for (uint32_t st = (issued > kStages ? issued - kStages : 0); st < issued; ++st)
                    mbar_wait(&full[st % kStages], (st / kStages) & 1, shape.limit);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer
            uint32_t step = 0, local = 0;
            bool ok = true;
            for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++local) {
                const uint32_t acc = local & 1, use = local >> 1;
                if (*abort_flag || !mbar_wait(&acc_empty[acc], (use & 1) ^ 1, shape.limit, abort_flag)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t d_tmem = tmem + acc * kAccColumns;
                for (uint32_t ks = 0; ks < shape.k_tiles; ++ks, ++step) {
                    const uint32_t s = step % kStages, round = step / kStages;
                    if (*abort_flag || !mbar_wait(&full[s], round & 1, shape.limit, abort_flag)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t a_addr = smem_u32(a_smem + s * kATileBytes);
                    const uint32_t b_addr = smem_u32(b_smem + s * kBTileBytes);
#pragma unroll
                    for (uint32_t kk = 0; kk < kBlockK / 32; ++kk)
                        mma_i8(d_tmem, smem_descriptor(a_addr + kk * 32), smem_descriptor(b_addr + kk * 32),
                               (ks | kk) != 0 ? 1u : 0u);
                    mma_commit(&empty[s]);  // frees the stage once these MMAs have read it
                }
                if (ok) mma_commit(&acc_full[acc]);  // accumulator complete
            }
            if (!ok) {
                *abort_flag = 1;
                record_error(shape.status, 2u);
            }
            mma_commit(drain);  // arrives once every MMA issued above has completed
            if (!mbar_wait(drain, 0, shape.limit)) record_error(shape.status, 8u);
        }
    } else {
        // ---------------- epilogue: warp w reads TMEM lanes 32*(w%4).. (rows of the tile)
        const uint32_t quarter = warp & 3;
        uint32_t local = 0;
        for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++local) {
            const uint32_t acc = local & 1, use = local >> 1;
            uint32_t m_tile, n_tile;
            tile_coords(tile, shape, m_tile, n_tile);
            const uint32_t row0 = m_tile * kBlockM, col0 = n_tile * kBlockN;
            bool have = !*abort_flag && mbar_wait(&acc_full[acc], use & 1, shape.limit, abort_flag);
            have = __all_sync(0xffffffffu, have);
            if (!have) {
                if (lane == 0) {
                    *abort_flag = 1;
                    record_error(shape.status, 4u);
                }
                break;
            }
            fence_after();
            const uint32_t row = row0 + quarter * 32 + lane;  // GEMM row of this lane
            const bool row_ok = row < shape.m;
            uint32_t op = 0, column = 0;
            uint64_t out_row = 0;
            if (row_ok) {
                if (epi.mode == kEpilogueConvert)
                    shape.rows.residue(row, op, column);
                else
                    out_row = shape.rows.row(row);
            }
            const uint32_t t_base = tmem + acc * kAccColumns + ((quarter * 32) << 16);
            epilogue_rows(epi, t_base, col0, shape.columns, row_ok, out_row, op, column, lane);
            // every tcgen05.ld of this warp has completed (tmem_load32 waits): release the accumulator
            fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[acc])) : "memory");
        }
    }
    __syncwarp();
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kAccColumns)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// Pair (2-CTA) variant: a cluster of two CTAs computes a 256 x 256 tile with
// tcgen05.mma.cta_group::2 (M = 256, N = 256). CTA rank r holds A rows
// [128r, 128r+128) and B columns [128r, 128r+128) of the tile in its own shared
// memory and rows [128r, 128r+128) of the accumulator in its own TMEM. Per MMA
// each SM reads half the B bytes of the single-CTA kernel, and each stage
// moves 32 KB per SM from L2 instead of 48 KB.
//   * both CTAs' TMA loads complete on the leader's (rank 0) full[s] barrier,
//     which the leader arms with both CTAs' bytes;
//   * the leader's single MMA thread commits to empty[s] / acc_full[a] in both
//     CTAs at once (tcgen05.commit ... multicast::cluster, mask 0b11);
//   * all eight epilogue warps of the pair release an accumulator on the
//     leader's acc_empty[a] (cluster-scope arrive).
constexpr uint32_t kPairStages = 7;  // 224 KB of ring: seven stages fit the 227 KB opt-in limit with the barriers
constexpr uint32_t kPairBlockN = 256;                      // columns per pair tile
constexpr uint32_t kPairBTileBytes = (kPairBlockN / 2) * kBlockK;  // 16 KB: this CTA's half of B
constexpr uint32_t kPairStageBytes = kATileBytes + kPairBTileBytes; // 32 KB per CTA
constexpr size_t kPairSmemBytes = size_t(kPairStages) * kPairStageBytes + 1024 + 256;
constexpr uint32_t kPairInstrDesc = (2u << 4) | ((kPairBlockN >> 3) << 17) | ((256u >> 4) << 24);

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    return rank;
}

__device__ __forceinline__ uint32_t leader_address(const void* local) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(local)), "r"(0));
    return remote;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t bar_cluster, int c0,
                                                 int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem_d, uint64_t desc_a, uint64_t desc_b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(desc_a), "l"(desc_b), "r"(kPairInstrDesc), "r"(accumulate)
        : "memory");
}

// arrive on the barrier at this shared-memory offset in both CTAs of the pair
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(uint16_t(3))
        : "memory");
}

// arrive on this CTA's barrier once the pair MMAs issued so far have completed
__device__ __forceinline__ void mma_commit_pair_local(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}

__device__ __forceinline__ void mbar_arrive_local(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait with cluster-scope acquire: data written by the other CTA of the pair before its
// release-arrive on this barrier is visible afterwards. Ends early once the abort flag is raised.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, long long limit,
                                                  const volatile uint32_t* abort) {
    const long long start = clock64();
    for (uint32_t i = 0;; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 63u) == 63u && (*abort || clock64() - start > limit)) return false;
    }
}

__device__ __forceinline__ uint32_t peer_address(const void* local) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(local)), "r"(1));
    return remote;
}

// this CTA's shared-memory word at the same offset in the other CTA of the pair
__device__ __forceinline__ uint32_t other_address(const void* local, uint32_t rank) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(local)), "r"(rank ^ 1u));
    return remote;
}

// Dynamic tile order: the leader's producer claims tile indices from a global counter (zeroed
// by the host before the launch) and hands each one to every role of both CTAs through a ring
// of kRing slots: tile_ring[slot] plus ring_full[slot] in each CTA, and ring_empty[slot] in the
// leader, which all kRingReaders readers arrive on once they have read the slot. An index at or
// past the tile count ends every role's loop. Claiming in order keeps the tiles in flight within
// one window of the raster order (one L2-sized group), whatever the pace of each pair.
constexpr uint32_t kRing = 4;
constexpr uint32_t kRingReaders = 1 /* peer producer */ + 1 /* leader MMA */ + 2 * kEpilogueWarps;

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    gemm_tc_pair_kernel(const __grid_constant__ CUtensorMap a_map, const __grid_constant__ CUtensorMap b_map,
                        TileShape shape, Epilogue epi) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* a_smem = smem;
    uint8_t* b_smem = smem + kPairStages * kATileBytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(b_smem + kPairStages * kPairBTileBytes);
    uint64_t* empty = full + kPairStages;
    uint64_t* acc_full = empty + kPairStages;  // [2]
    uint64_t* acc_empty = acc_full + 2;        // [2] (leader's are used)
    uint64_t* drain = acc_empty + 2;
    uint64_t* ring_full = drain + 1;           // [kRing]
    uint64_t* ring_empty = ring_full + kRing;  // [kRing] (leader's are used)
    uint32_t* tile_ring = reinterpret_cast<uint32_t*>(ring_empty + kRing);  // [kRing]
    uint32_t* tmem_slot = tile_ring + kRing;
    volatile uint32_t* abort_flag = tmem_slot + 1;

    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t rank = cluster_rank();
    const long long limit = shape.limit;
    // Raises the abort flag in both CTAs of the pair, so that every role of both ends its waits at
    // once (the other CTA stays resident until the final cluster barrier, so the store is safe).
    auto raise_abort = [&](uint32_t bit) {
        *abort_flag = 1;
        asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(other_address(const_cast<uint32_t*>(abort_flag), rank)),
                     "r"(1u)
                     : "memory");
        record_error(shape.status, bit);
    };
    const bool leader = rank == 0;
    const uint32_t tiles = shape.m_tiles * shape.n_tiles;  // m_tiles counts 256-row pair tiles

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < kPairStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (uint32_t a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 2 * kEpilogueWarps);
        }
        for (uint32_t i = 0; i < kRing; ++i) {
            mbar_init(&ring_full[i], 1);
            mbar_init(&ring_empty[i], kRingReaders);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * kAccColumns)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    fence_before();
    cluster_sync();  // barriers and TMEM of both CTAs ready before any cross-CTA traffic
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t ring_release = leader_address(&ring_empty[0]);  // + slot * 8

    // Reads ring slot i (every reader): the tile index, or `tiles` after a timeout or an abort.
    auto read_ring = [&](uint32_t i, bool all_lanes_wait) -> uint32_t {
        const uint32_t slot = i % kRing, round = i / kRing;
        bool ok = true;
        if (all_lanes_wait || lane == 0) ok = !*abort_flag && mbar_wait_cluster(&ring_full[slot], round & 1, limit, abort_flag);
        uint32_t tile = ok ? tile_ring[slot] : tiles;
        if (!ok) raise_abort(256u);
        return tile;
    };

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer (both CTAs): own A half and B half, leader's barrier
            uint32_t step = 0;
            bool ok = true, withheld = false;
            for (uint32_t i = 0; ok && !withheld; ++i) {
                uint32_t tile;
                if (leader) {  // claim the next tile and publish it to both CTAs
                    const uint32_t slot = i % kRing, round = i / kRing;
                    if (*abort_flag || !mbar_wait_cluster(&ring_empty[slot], (round & 1) ^ 1, limit, abort_flag)) {
                        ok = false;
                        // release every reader of this and later slots: they see an end index
                        tile = tiles;
                    } else {
                        tile = atomicAdd(shape.tile_counter, 1u);
                    }
                    if (tile > tiles) tile = tiles;
                    tile_ring[slot] = tile;
                    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(peer_address(&tile_ring[slot])), "r"(tile)
                                 : "memory");
                    mbar_arrive_cluster(peer_address(&ring_full[slot]));
                    mbar_arrive_local(&ring_full[slot]);
                } else {
                    tile = read_ring(i, true);
                    mbar_arrive_cluster(ring_release + (i % kRing) * sizeof(uint64_t));
                }
                if (tile >= tiles) break;
                uint32_t m_tile, n_tile;
                tile_coords(tile, shape, m_tile, n_tile);
                const uint32_t row0 = m_tile * 256 + rank * kBlockM;
                const uint32_t col0 = n_tile * kPairBlockN + rank * (kPairBlockN / 2);
                const uint32_t a_row = uint32_t(shape.rows.row(row0));  // 128 consecutive operand rows
                for (uint32_t ks = 0; ks < shape.k_tiles; ++ks, ++step) {
                    const uint32_t s = step % kPairStages, round = step / kPairStages;
                    if (leader && blockIdx.x == 0 && step == shape.withheld) {  // diagnostics: never armed
                        withheld = true;
                        break;
                    }
                    if (*abort_flag || !mbar_wait(&empty[s], (round & 1) ^ 1, limit, abort_flag)) {
                        ok = false;
                        break;
                    }
                    if (leader) mbar_expect_tx(&full[s], 2 * kPairStageBytes);
                    const uint32_t bar = leader_address(&full[s]);
                    tma_load_2d_pair(a_smem + s * kATileBytes, &a_map, bar, int(ks * kBlockK), int(a_row));
                    tma_load_2d_pair(b_smem + s * kPairBTileBytes, &b_map, bar, int(ks * kBlockK), int(col0));
                }
            }
            if (!ok) raise_abort(16u);
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ---------------- MMA issuer (leader only)
            uint32_t step = 0, local = 0;
            bool ok = true;
            for (uint32_t i = 0; ok; ++i, ++local) {
                const uint32_t tile = read_ring(i, true);
                mbar_arrive_local(&ring_empty[i % kRing]);
                if (tile >= tiles) break;
                const uint32_t acc = local & 1, use = local >> 1;
                if (*abort_flag || !mbar_wait(&acc_empty[acc], (use & 1) ^ 1, limit, abort_flag)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t d_tmem = tmem + acc * kAccColumns;
                for (uint32_t ks = 0; ks < shape.k_tiles; ++ks, ++step) {
                    const uint32_t s = step % kPairStages, round = step / kPairStages;
                    if (*abort_flag || !mbar_wait(&full[s], round & 1, limit, abort_flag)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t a_addr = smem_u32(a_smem + s * kATileBytes);
                    const uint32_t b_addr = smem_u32(b_smem + s * kPairBTileBytes);
#pragma unroll
                    for (uint32_t kk = 0; kk < kBlockK / 32; ++kk)
                        mma_i8_pair(d_tmem, smem_descriptor(a_addr + kk * 32), smem_descriptor(b_addr + kk * 32),
                                    (ks | kk) != 0 ? 1u : 0u);
                    mma_commit_pair(&empty[s]);  // frees stage s in both CTAs
                }
                if (ok) mma_commit_pair(&acc_full[acc]);
            }
            if (!ok) raise_abort(32u);
            mma_commit_pair_local(drain);  // every tcgen05 op here is cta_group::2
            if (!mbar_wait(drain, 0, limit)) raise_abort(64u);
        }
    } else {
        // ---------------- epilogue: this CTA's 128 rows of each pair tile
        const uint32_t quarter = warp & 3;
        const uint32_t release = leader_address(&acc_empty[0]);
        for (uint32_t i = 0, local = 0;; ++i, ++local) {
            uint32_t tile = read_ring(i, false);
            tile = __shfl_sync(0xffffffffu, tile, 0);
            if (lane == 0) {
                if (leader)
                    mbar_arrive_local(&ring_empty[i % kRing]);
                else
                    mbar_arrive_cluster(ring_release + (i % kRing) * sizeof(uint64_t));
            }
            if (tile >= tiles) break;
            const uint32_t acc = local & 1, use = local >> 1;
            uint32_t m_tile, n_tile;
            tile_coords(tile, shape, m_tile, n_tile);
            const uint32_t row0 = m_tile * 256 + rank * kBlockM, col0 = n_tile * kPairBlockN;
            bool have = !*abort_flag && mbar_wait(&acc_full[acc], use & 1, limit, abort_flag);
            have = __all_sync(0xffffffffu, have);
            if (!have) {
                if (lane == 0) raise_abort(128u);
                break;
            }
            fence_after();
            const uint32_t row = row0 + quarter * 32 + lane;
            const bool row_ok = row < shape.m;
            uint32_t op = 0, column = 0;
            uint64_t out_row = 0;
            if (row_ok) {
                if (epi.mode == kEpilogueConvert)
                    shape.rows.residue(row, op, column);
                else
                    out_row = shape.rows.row(row);
            }
            const uint32_t t_base = tmem + acc * kAccColumns + ((quarter * 32) << 16);
            epilogue_rows(epi, t_base, col0, shape.columns, row_ok, out_row, op, column, lane);
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(release + acc * sizeof(uint64_t));
        }
    }
    __syncwarp();
    // After an abort, TMA loads of either CTA may still be in flight (a producer that stopped does
    // not know which of the leader's stage barriers will complete): one thread holds this CTA, and
    // through the barrier below its peer, until they have landed.
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) abort_drain();
    fence_before();
    cluster_sync();  // the leader's MMAs have drained and no peer accesses remain
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kAccColumns)
                     : "memory");
    }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult status{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &status) == cudaSuccess &&
            status == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(ptr);
    }
    return fn;
}

}  // namespace

uint32_t* tensor_gemm_error_flag() {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_tc_error) != cudaSuccess) return nullptr;
    return static_cast<uint32_t*>(ptr);
}

bool prepare_gemm_tensor(TensorGemmPlan& plan, const uint8_t* a, uint64_t a_pitch, RowMap rows, uint32_t m,
                         const uint8_t* b, uint32_t columns, uint32_t k_bytes, std::string& why) {
    plan.ready = false;
    EncodeTiled encode = encoder();
    if (!encode) {
        why = "cuTensorMapEncodeTiled unavailable";
        return false;
    }
    if (k_bytes < kBlockK || k_bytes % 16 || a_pitch % 16 || a_pitch < k_bytes) {
        why = "K must be >= 128 bytes with 16-byte rows";
        return false;
    }
    if (reinterpret_cast<uintptr_t>(a) % 16 || reinterpret_cast<uintptr_t>(b) % 16) {
        why = "operands must be 16-byte aligned";
        return false;
    }
    if (columns < kBlockN) {
        why = "fewer than 256 output columns";
        return false;
    }
    uint32_t slab = m;
    if (rows.mode == kRowsSplit) {
        slab = rows.n_sub;
        if (m != 2 * rows.n || rows.first != 0 || rows.span != rows.n_sub || rows.t_first != 0 ||
            rows.t_count != rows.split) {
            why = "split row map expects both whole operands";
            return false;
        }
    } else if (rows.first != 0) {
        why = "linear row map must start at row 0";
        return false;
    }
    if (slab < kBlockM || (rows.mode == kRowsSplit && slab % kBlockM)) {
        why = "fewer than 128 rows per transform";
        return false;
    }
    // A: m operand rows of k_bytes (row pitch a_pitch); split-major operands make every
    // 128-row tile of a split row map one contiguous box
    const cuuint64_t a_dims[2] = {k_bytes, m};
    const cuuint64_t a_strides[1] = {a_pitch};
    const cuuint32_t a_box[2] = {kBlockK, kBlockM};
    const cuuint32_t unit[2] = {1, 1};
    CUresult ra = encode(&plan.a_map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(a), a_dims, a_strides,
                         a_box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    const cuuint64_t b_dims[2] = {k_bytes, columns};
    const cuuint64_t b_strides[1] = {k_bytes};
    const cuuint32_t b_box[2] = {kBlockK, kBlockN};
    CUresult rb = encode(&plan.b_map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(b), b_dims, b_strides,
                         b_box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    const cuuint32_t b_half_box[2] = {kBlockK, kPairBlockN / 2};
    CUresult rh = encode(&plan.b_map_half, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(b), b_dims,
                         b_strides, b_half_box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (ra != CUDA_SUCCESS || rb != CUDA_SUCCESS || rh != CUDA_SUCCESS) {
        why = "tensor map encoding failed";
        return false;
    }
    if (cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(gemm_tc_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kPairSmemBytes)) != cudaSuccess) {
        cudaGetLastError();
        why = "cannot reserve shared memory";
        return false;
    }
    plan.m = m;
    plan.columns = columns;
    plan.k_bytes = k_bytes;
    plan.m_tiles = (m + kBlockM - 1) / kBlockM;
    plan.n_tiles = (columns + kBlockN - 1) / kBlockN;
    plan.k_tiles = (k_bytes + kBlockK - 1) / kBlockK;
    plan.rows = rows;
    plan.a_tile_bytes = uint64_t(kBlockM) * k_bytes;
    plan.error_flag = tensor_gemm_error_flag();
    if (!plan.tile_counter) {  // callers that keep GEMMs of one plan on one stream may bind their own
        void* counter = nullptr;
        if (cudaGetSymbolAddress(&counter, g_tile_counter) != cudaSuccess) {
            cudaGetLastError();
            why = "no tile counter";
            return false;
        }
        plan.tile_counter = static_cast<uint32_t*>(counter);
    }
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    plan.sm_count = sms > 0 ? uint32_t(sms) : 148;
    // CTA pairs need 256-row slabs; NEGACYCLIC_GEMM_PAIRS=0 selects the single-CTA kernel
    const char* pairs_env = getenv("NEGACYCLIC_GEMM_PAIRS");
    plan.pairs = !(pairs_env && pairs_env[0] == '0') && plan.sm_count >= 2 &&
                 (rows.mode == kRowsLinear || slab % 256 == 0);
    plan.ready = true;
    return true;
}

bool gemm_tensor_accepts(const TensorGemmPlan& plan, const RowMap& rows, uint32_t m) {
    if (!plan.ready || rows.mode != plan.rows.mode) return false;
    if (rows.mode == kRowsSplit)
        return rows.span % kBlockM == 0 && rows.first % kBlockM == 0 && rows.first + rows.span <= plan.rows.n_sub &&
               rows.t_first + rows.t_count <= plan.rows.split && m % (rows.t_count * rows.span) == 0 &&
               rows.op_first + m / (rows.t_count * rows.span) <= 2;
    return uint64_t(rows.first) + m <= plan.m;
}

void launch_gemm_tensor(const TensorGemmPlan& plan, const Epilogue& epilogue, cudaStream_t stream, const RowMap& rows,
                        uint32_t m, bool allow_pairs, long long limit_cycles, uint32_t withheld) {
    const bool pairs = allow_pairs && plan.pairs && (rows.mode == kRowsLinear || rows.span % 256 == 0);
    const uint32_t rows_per_tile = pairs ? 256 : kBlockM;
    const uint32_t m_tiles = (m + rows_per_tile - 1) / rows_per_tile;
    // largest raster group whose A tiles fit comfortably in L2 (~48 MB)
    uint64_t group = (48ull << 20) / (plan.a_tile_bytes * (pairs ? 2 : 1));
    group = group < 4 ? 4 : (group > 64 ? 64 : group);
    TileShape shape{m,      plan.columns,       plan.k_tiles,
                    m_tiles, plan.n_tiles,      uint32_t(group),
                    rows,    plan.tile_counter, epilogue.status,
                    limit_cycles > 0 ? limit_cycles : kDefaultLimitCycles, withheld};
    const uint32_t tiles = m_tiles * plan.n_tiles;
    if (pairs) {
        const uint32_t max_pairs = plan.sm_count / 2;
        const uint32_t grid = 2 * (tiles < max_pairs ? tiles : max_pairs);
        cudaMemsetAsync(plan.tile_counter, 0, sizeof(uint32_t), stream);
        gemm_tc_pair_kernel<<<grid, kThreads, kPairSmemBytes, stream>>>(plan.a_map, plan.b_map_half, shape, epilogue);
        return;
    }
    const uint32_t grid = tiles < plan.sm_count ? tiles : plan.sm_count;
    gemm_tc_kernel<<<grid, kThreads, kSmemBytes, stream>>>(plan.a_map, plan.b_map, shape, epilogue);
}

void launch_gemm_tensor(const TensorGemmPlan& plan, const Epilogue& epilogue, cudaStream_t stream, const RowMap& rows,
                        uint32_t m) {
    launch_gemm_tensor(plan, epilogue, stream, rows, m, true, 0, kNoWithheldStep);
}

void launch_gemm_tensor(const TensorGemmPlan& plan, const Epilogue& epilogue, cudaStream_t stream) {
    launch_gemm_tensor(plan, epilogue, stream, plan.rows, plan.m);
}

}  // namespace negacyclic
