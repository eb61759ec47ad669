// Byte-sliced u8 x u8 -> s32 GEMM on the 5th-generation tensor cores (sm_100a).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>

#include "kernels.cuh"

namespace negacyclic {

struct TensorGemmPlan {
    CUtensorMap a_map;   // 2-D view of A: (K bytes, rows),          box (128, 128),   128B swizzle
    CUtensorMap b_map;   // 2-D view of B: (K bytes, columns),       box (128, 256),   128B swizzle
    CUtensorMap b_map_half;  // same view, box (128, 128): one CTA's half of a pair tile
    uint32_t m = 0, columns = 0, k_bytes = 0;
    uint32_t m_tiles = 0, n_tiles = 0, k_tiles = 0;
    RowMap rows{};
    uint32_t* error_flag = nullptr;  // device word set when a pipeline wait times out
    uint32_t* tile_counter = nullptr;  // device word the CTA-pair kernel claims tiles from; GEMMs that
                                       // share one may not run at the same time
    uint32_t sm_count = 148;          // persistent grid size
    uint64_t a_tile_bytes = 0;        // bytes of one 128-row A tile (raster group sizing)
    bool pairs = false;               // 2-CTA (cta_group::2) 256x256 tiles
    bool ready = false;
};

// Builds the tensor maps; false (with `why`) when the shape is outside what the
// kernel handles (then the SIMT kernel is used).
bool prepare_gemm_tensor(TensorGemmPlan& plan, const uint8_t* a, uint64_t a_pitch, RowMap rows, uint32_t m,
                         const uint8_t* b, uint32_t columns, uint32_t k_bytes, std::string& why);

void launch_gemm_tensor(const TensorGemmPlan& plan, const Epilogue& epilogue, cudaStream_t stream);

// A launch over part of the rows (a chunk of coefficients): `rows`/`m` describe the chunk
// within the shape the plan was prepared for (see gemm_tensor_accepts).
void launch_gemm_tensor(const TensorGemmPlan& plan, const Epilogue& epilogue, cudaStream_t stream, const RowMap& rows,
                        uint32_t m);
// allow_pairs = false forces the single-CTA kernel (diagnostics and tests). limit_cycles bounds
// every pipeline wait (0 = the default, about 2 s of SM clock). withheld (diagnostics only): the
// producer of the first CTA (pair) stops before this pipeline step, so that its consumer's wait
// runs out; kNoWithheldStep in normal use.
constexpr uint32_t kNoWithheldStep = 0xffffffffu;
void launch_gemm_tensor(const TensorGemmPlan& plan, const Epilogue& epilogue, cudaStream_t stream, const RowMap& rows,
                        uint32_t m, bool allow_pairs, long long limit_cycles, uint32_t withheld);
bool gemm_tensor_accepts(const TensorGemmPlan& plan, const RowMap& rows, uint32_t m);

// Device word that records pipeline-wait timeouts of the tensor GEMM (0 = none).
uint32_t* tensor_gemm_error_flag();

}  // namespace negacyclic
