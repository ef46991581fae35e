// ABI types of the platform's polymul/negacyclic kernel contract.
//
// The drop-in contract is the reference's generated header (fherma.h:13-47 in the reference):
// a harness compiled against that header links against this library, so the types below must
// have the same members, in the same order, with the same types, and the three entry points
// keep C++ linkage. This file restates that contract for this build; it is not a copy of the
// generated file.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace fherma {

// A dense tensor: shape and row-major elements (fherma.h:15-25).
template <class T>
struct Tensor {
    std::vector<int64_t> shape;
    std::vector<T> data;

    int64_t count() const {
        int64_t n = 1;
        for (int64_t d : shape) n *= d;
        return n;
    }
};

// The problem point: ring degree N, modulus width W in bits, L = (W + 31) / 32 limbs,
// and q as L little-endian u32 limbs (fherma.h:27-32).
struct Point {
    uint32_t N = 0;
    uint32_t W = 0;
    uint32_t L = 0;
    Tensor<uint32_t> q;
};

// Operands a and b, each N x L little-endian u32 limbs, coefficient-major (fherma.h:34-37).
struct Inputs {
    Tensor<uint32_t> a;
    Tensor<uint32_t> b;
};

// The product c, N x L limbs (fherma.h:39-41).
struct Outputs {
    Tensor<uint32_t> c;
};

}  // namespace fherma

// Setup, not timed by the harness (fherma.h:45). Throws std::runtime_error on a bad point.
void* fherma_init(const fherma::Point& p);
// c = a * b mod (X^N + 1, q), host buffers in and out (fherma.h:46). Throws on bad sizes.
fherma::Outputs fherma_run(void* state, const fherma::Inputs& in);
// Releases the state; a null state is a no-op (fherma.h:47).
void fherma_free(void* state);
