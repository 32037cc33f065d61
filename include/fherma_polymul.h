// fherma_polymul.h -- the reference's solution interface, served by libpolymul.
//
// The reference solution is three C++ functions over a handful of value types
// (fherma.h:14-46 of ilyausmanov2015/fherma-polymul-baseline, generated from the
// FHERMA task polymul/negacyclic@1.0.0).  A harness compiled against that header
// links libfherma_polymul.so instead of the reference's solve.cu; for that the
// types below must have the same members, in the same order, with the same
// C++ types, and the functions the same C++ signatures.
//
// Semantics (as the reference's rns/solve.cu:581-854 gives them):
//   fherma_init  -- untimed set-up for one point (N, W, L, q); returns an opaque
//                   state; throws std::runtime_error outside coverage.
//   fherma_run   -- c = a * b mod (X^N + 1, q), a fresh N x L tensor; inputs are
//                   only read during the call; throws std::runtime_error on failure.
//   fherma_free  -- releases the state.
// Coverage here is wider than the reference's (q = 2^868 - c, N <= 32768):
// any odd q with at most W <= 32*L bits, N a power of two in [2, 65536], L even.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace fherma {

template <class T>
struct Tensor {
    std::vector<int64_t> shape;
    std::vector<T> data;  // row-major

    int64_t count() const {
        int64_t n = 1;
        for (int64_t d : shape) n *= d;
        return n;
    }
};

struct Point {
    uint32_t N = 0;       // ring dimension
    uint32_t W = 0;       // bit width of q
    uint32_t L = 0;       // 32-bit words per coefficient
    Tensor<uint32_t> q;   // L words, least significant first
};

struct Inputs {
    Tensor<uint32_t> a;   // N x L
    Tensor<uint32_t> b;   // N x L
};

struct Outputs {
    Tensor<uint32_t> c;   // N x L
};

}  // namespace fherma

void* fherma_init(const fherma::Point& p);
fherma::Outputs fherma_run(void* state, const fherma::Inputs& in);
void fherma_free(void* state);
