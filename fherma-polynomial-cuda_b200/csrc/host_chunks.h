// Chunk lists of the streamed host path (negacyclic_run, run_begin/run_finish): which pieces of
// the operands go to the device in which order, and in which pieces the result comes back.
// Host-only and free of CUDA types, so that tests/native/host_chunks_check.cpp checks the lists
// on the CPU for every shape.
//
// In: rows of at least 1 KB go in transform order: a chunk is part of transform t, positions j
// in [j0, j0 + span), i.e. coefficients s*j + t (one 2-D copy per operand), so the forward NTTs
// of transform t run while later transforms are still being copied in. Narrower rows go as
// contiguous coefficient ranges of operand a, then of operand b, so that a's forward NTTs run
// while b is still being copied in.
// Out: contiguous coefficient ranges; each chunk's copy-out overlaps the next chunk's CRT GEMM
// and reduction.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace negacyclic {

constexpr uint32_t kMaxHostChunks = 16;  // events per direction a plan keeps

struct ChunkShape {
    uint32_t n, n_sub, split, limbs;
    uint32_t chunks;  // host_chunks(): 1, or max(8, s)
};

struct InChunk {  // transform t, positions j in [j0, j0 + span): coefficients s*j + t
    uint32_t t, j0, span;
    uint32_t op = kBothOperands;  // operand 0 (a) or 1 (b), or both
    static constexpr uint32_t kBothOperands = 2;
};
struct OutChunk {  // coefficients [first, first + count)
    uint32_t first, count;
};

// Host products stream in about max(8, s) chunks each way once each chunk keeps 128-row GEMM
// tiles (N' >= 1024, N >= 8192); smaller products go in one piece each way.
inline uint32_t host_chunks(uint32_t n, uint32_t n_sub, uint32_t split) {
    return (n_sub >= 1024 && n >= 8192) ? std::max(8u, split) : 1u;
}

// Rows of at least 1 KB: chunks carry enough work that finer chunks near the ends (and one
// transpose per output chunk) pay for their extra launches. Narrower rows keep equal chunks.
inline bool wide_rows(const ChunkShape& s) { return s.limbs >= 256; }

// Transform order needs rows gathered with a stride of s rows, by the copy engine as a 2-D copy
// or by the host team while it packs pageable operands. Both pay only for rows of 1 KB or more:
// a 2-D copy of 220-byte rows ran at a third of the link rate, and the team gathering 220-byte
// rows packed at 20 GB/s against 55 GB/s for contiguous ranges (N=65536, L=55).
inline bool transform_ordered_input(const ChunkShape& s) {
    return s.chunks > 1 && s.split > 1 && wide_rows(s);  // chunks >= split when chunked
}

// Chunks of about `target` bytes out of `bytes`: a power of two in [2, min(most, limit)].
inline uint32_t chunk_count(size_t bytes, size_t target, uint32_t most, uint32_t limit) {
    uint32_t count = 2;
    while (count * 2 <= std::min(most, limit) && bytes / (count * 2) >= target) count *= 2;
    return std::max(1u, std::min(count, std::min(most, limit)));
}

// Chunk lists of a streamed host product (at most kMaxHostChunks each way).
// In, transform-ordered: `parts` chunks per transform, the last transform cut finer, so that
// little conversion is left once the link has delivered everything. In, coefficient-ordered,
// wide rows: equal coefficient ranges of both operands, the last one cut in four; narrow rows:
// equal ranges of operand a, then of operand b. Out, wide rows: coefficient ranges growing from
// a quarter of a chunk, so the copy-out starts soon after the last inverse NTT; narrow rows:
// equal ranges of about 1 MB.
inline void stream_chunks(const ChunkShape& s, bool ordered, std::vector<InChunk>& in, std::vector<OutChunk>& out) {
    const uint32_t split = s.split, n_sub = s.n_sub, per = s.n / s.chunks;
    constexpr uint32_t kMax = kMaxHostChunks;
    in.clear();
    out.clear();
    if (s.chunks == 1) {  // small product: one piece each way
        in.push_back(InChunk{0, 0, s.n});
        out.push_back(OutChunk{0, s.n});
        return;
    }
    if (ordered) {
        const uint32_t parts = s.chunks / split;
        uint32_t tail = parts;  // power of two, spans of >= 256 rows, within the event budget
        while (tail * 2 <= 4 * parts && (split - 1) * parts + tail * 2 <= kMax && n_sub / (tail * 2) >= 256) tail *= 2;
        for (uint32_t t = 0; t < split; ++t) {
            const uint32_t p = t + 1 == split ? tail : parts, span = n_sub / p;
            for (uint32_t k = 0; k < p; ++k) in.push_back(InChunk{t, k * span, span});
        }
    } else if (wide_rows(s)) {
        const uint32_t quarter = per / 4;
        const bool cut = quarter / split >= 256 && s.chunks + 3 <= kMax;
        for (uint32_t k = 0; k + 1 < s.chunks; ++k) in.push_back(InChunk{0, k * per, per});
        if (cut)
            for (uint32_t k = 0; k < 4; ++k) in.push_back(InChunk{0, (s.chunks - 1) * per + k * quarter, quarter});
        else
            in.push_back(InChunk{0, (s.chunks - 1) * per, per});
    } else {
        // narrow rows: operand a, then operand b, each in coefficient ranges of about 1 MB (at
        // least two per operand, and at least 256 positions of every transform each), so that a's
        // conversion and forward NTTs run while b is still on the way. Small copies carry fixed
        // costs: 0.46 MB host-to-device copies ran at 23 GB/s against 55 for large ones (N=32768,
        // L=28).
        const uint32_t count = chunk_count(size_t(s.n) * s.limbs * 4, 1u << 20, std::min(s.chunks, kMax / 2),
                                           n_sub / 256);
        const uint32_t span = s.n / count;
        for (uint32_t op = 0; op < 2; ++op)
            for (uint32_t k = 0; k < count; ++k) in.push_back(InChunk{0, k * span, span, op});
    }
    if (wide_rows(s)) {  // per/4, per/4, per/2, then whole chunks: two chunks more than the plain split
        uint32_t first = 0, size = (per / 4 >= 256 && s.chunks + 2 <= kMax) ? per / 4 : per;
        for (uint32_t k = 0; first < s.n; ++k) {
            const uint32_t count = std::min(size, s.n - first);
            out.push_back(OutChunk{first, count});
            first += count;
            if (k >= 1 && size < per) size *= 2;  // per/4, per/4, per/2, per, per, ...
        }
        return;
    }
    // narrow rows: about 1 MB of result per chunk, at least 256 coefficients each
    const uint32_t count = chunk_count(size_t(s.n) * s.limbs * 4, 1u << 20, s.chunks, s.n / 256);
    for (uint32_t k = 0; k < count; ++k) out.push_back(OutChunk{k * (s.n / count), s.n / count});
}

}  // namespace negacyclic
