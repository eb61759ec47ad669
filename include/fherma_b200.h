// fherma_b200.h — the reference plugin's C++ entry points, provided by
// libfherma_negacyclic.so on top of the C ABI in negacyclic.h.
//
// The types are layout-compatible with the FHERMA-generated header the
// reference is written against (src/fherma.h:13-48: Tensor<T>{shape, data}
// row-major, Point{N, W, L, q}, Inputs{a, b}, Outputs{c}); the platform's
// harness (src/main.cpp) compiles against its own generated copy and links
// this library unchanged. Errors are thrown as std::runtime_error, as the
// reference does (src/solve.cu:32-34, 506-507, 579).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#ifndef FHERMA_TYPES_DEFINED
#define FHERMA_TYPES_DEFINED
namespace fherma {

template <class T>
struct Tensor {
    std::vector<int64_t> shape;  // {N, L} for operands, {L} for q
    std::vector<T> data;         // row-major

    int64_t count() const {
        int64_t total = 1;
        for (int64_t d : shape) total *= d;
        return total;
    }
};

struct Point {
    uint32_t N = 0;  // ring degree, a power of two
    uint32_t W = 0;  // bit width of q; L == (W + 31) / 32
    uint32_t L = 0;  // limbs per coefficient
    Tensor<uint32_t> q;
};

struct Inputs {
    Tensor<uint32_t> a;
    Tensor<uint32_t> b;
};

struct Outputs {
    Tensor<uint32_t> c;
};

}  // namespace fherma
#endif

void* fherma_init(const fherma::Point& p);
fherma::Outputs fherma_run(void* state, const fherma::Inputs& in);
void fherma_free(void* state);
