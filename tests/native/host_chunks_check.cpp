// CPU check of the streamed host path's chunk lists (fherma-polynomial-cuda_b200/csrc/host_chunks.h),
// built and run by tests/test_host_chunks.py, for every N = 2^0..2^17, every ring split s with
// N/s <= 8192, and limb counts on both sides of the wide-row threshold:
//  * at most kMaxHostChunks chunks each way (the plan keeps that many events per direction);
//  * the input chunks cover every coefficient of both operands exactly once;
//  * coefficient-range chunks start and end on multiples of s (host_begin converts positions
//    j in [first/s, (first+count)/s) of every transform), transform chunks stay inside one
//    transform, and narrow-row chunks send all of operand a before operand b;
//  * the output chunks tile [0, N) in order, on multiples of s where each chunk transposes its own
//    coefficients (wide rows).
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../fherma-polynomial-cuda_b200/csrc/host_chunks.h"

using namespace negacyclic;

static int failures = 0;
static ChunkShape current;
#define EXPECT(cond)                                                                                       \
    do {                                                                                                   \
        if (!(cond)) {                                                                                     \
            if (failures < 20)                                                                             \
                std::fprintf(stderr, "N=%u s=%u L=%u chunks=%u: %s\n", current.n, current.split,            \
                             current.limbs, current.chunks, #cond);                                        \
            ++failures;                                                                                    \
        }                                                                                                  \
    } while (0)

static void check(const ChunkShape& s) {
    current = s;
    std::vector<InChunk> in;
    std::vector<OutChunk> out;
    const bool ordered = transform_ordered_input(s);
    stream_chunks(s, ordered, in, out);
    EXPECT(!in.empty() && in.size() <= kMaxHostChunks);
    EXPECT(!out.empty() && out.size() <= kMaxHostChunks);
    std::vector<uint8_t> seen(size_t(2) * s.n, 0);
    uint32_t last_op = 0;
    for (const InChunk& c : in) {
        EXPECT(c.span > 0);
        EXPECT(c.op <= InChunk::kBothOperands);
        const uint32_t op_first = c.op == InChunk::kBothOperands ? 0 : c.op;
        const uint32_t op_count = c.op == InChunk::kBothOperands ? 2 : 1;
        if (ordered) {  // transform t, positions [j0, j0 + span)
            EXPECT(c.op == InChunk::kBothOperands);
            EXPECT(c.t < s.split && uint64_t(c.j0) + c.span <= s.n_sub);
            for (uint32_t op = op_first; op < op_first + op_count; ++op)
                for (uint32_t j = c.j0; j < c.j0 + c.span && j < s.n_sub; ++j) ++seen[size_t(op) * s.n + size_t(s.split) * j + c.t];
        } else {  // coefficients [j0, j0 + span)
            EXPECT(c.t == 0 && uint64_t(c.j0) + c.span <= s.n);
            EXPECT(c.j0 % s.split == 0 && c.span % s.split == 0);
            if (c.op != InChunk::kBothOperands) {  // operand a's chunks all come first
                EXPECT(c.op >= last_op);
                last_op = c.op;
            }
            for (uint32_t op = op_first; op < op_first + op_count; ++op)
                for (uint32_t i = c.j0; i < c.j0 + c.span && i < s.n; ++i) ++seen[size_t(op) * s.n + i];
        }
    }
    bool once = true;
    for (uint8_t x : seen) once = once && x == 1;
    EXPECT(once);
    uint32_t next = 0;
    for (const OutChunk& c : out) {
        EXPECT(c.first == next && c.count > 0);
        if (wide_rows(s) && s.chunks > 1) EXPECT(c.first % s.split == 0 && c.count % s.split == 0);
        next = c.first + c.count;
    }
    EXPECT(next == s.n);
}

int main() {
    const uint32_t limb_counts[] = {1, 2, 28, 55, 100, 255, 256, 300, 868, 1747, 3000};
    int shapes = 0;
    for (uint32_t log_n = 0; log_n <= 17; ++log_n) {
        const uint32_t n = 1u << log_n;
        for (uint32_t split = 1; split <= 16 && split <= n; split *= 2) {
            const uint32_t n_sub = n / split;
            if (n_sub > 8192) continue;
            for (uint32_t limbs : limb_counts) {
                check(ChunkShape{n, n_sub, split, limbs, host_chunks(n, n_sub, split)});
                ++shapes;
            }
        }
    }
    std::printf("host chunks check: %d shapes, %d failures\n", shapes, failures);
    return failures ? 1 : 0;
}
