// fherma_init / fherma_run / fherma_free over the C ABI (include/negacyclic.h).
//
// Behaviour follows the reference's plugin (src/solve.cu:503-614):
//  * init validates the point (N a power of two, L == (W+31)/32) and builds
//    parameter-only state; no operand-dependent work (README.md:40);
//  * run checks operand sizes, returns a freshly allocated Outputs{c} of shape
//    {N, L}, and finishes all work before returning;
//  * failures throw std::runtime_error with the library's message.
// Compile with -DFHERMA_TYPES_DEFINED and the platform's fherma.h included
// first to use the generated types instead of include/fherma_b200.h's.
#include <stdexcept>
#include <string>

#include "../../include/fherma_b200.h"
#include "../../include/negacyclic.h"

namespace {

struct State {
    negacyclic_plan* plan = nullptr;
    uint32_t n = 0, limbs = 0;
};

[[noreturn]] void raise(const char* what) {
    throw std::runtime_error(std::string(what) + ": " + negacyclic_last_error());
}

}  // namespace

void* fherma_init(const fherma::Point& point) {
    if (point.q.data.size() != point.L) throw std::runtime_error("q must hold L words");
    auto* state = new State;
    state->n = point.N;
    state->limbs = point.L;
    if (negacyclic_init(point.N, point.W, point.L, point.q.data.data(), nullptr, &state->plan) != NEGACYCLIC_OK) {
        delete state;
        raise("fherma_init");
    }
    // the harness passes pageable std::vectors: page-locked staging is made here, not in the timed run
    if (negacyclic_prepare_host(state->plan) != NEGACYCLIC_OK) {
        negacyclic_free(state->plan);
        delete state;
        raise("fherma_init");
    }
    return state;
}

fherma::Outputs fherma_run(void* opaque, const fherma::Inputs& in) {
    auto* state = static_cast<State*>(opaque);
    const size_t count = size_t(state->n) * state->limbs;
    if (in.a.data.size() != count || in.b.data.size() != count) throw std::runtime_error("wrong input size");
    // the device computes while the output vector is allocated and zero-filled here
    if (negacyclic_run_begin(state->plan, in.a.data.data(), in.b.data.data()) != NEGACYCLIC_OK)
        raise("fherma_run");
    fherma::Outputs out;
    out.c.shape = {int64_t(state->n), int64_t(state->limbs)};
    out.c.data.resize(count);
    if (negacyclic_run_finish(state->plan, out.c.data.data()) != NEGACYCLIC_OK) raise("fherma_run");
    return out;
}

void fherma_free(void* opaque) {
    auto* state = static_cast<State*>(opaque);
    if (!state) return;
    negacyclic_free(state->plan);
    delete state;
}
