// Shared constants and plain-old-data structures for the negacyclic product library.
//
// The product c = a*b mod (X^N + 1, q) runs in the residue number system of a fixed set of
// 62-bit primes p = 2^62 - m with p = 1 (mod 2^17), so one prime set and one twiddle table
// serve every ring degree N <= 2^16 and every modulus width. The reference searches primes
// per N (solve.cu:1174-1204); any prime set whose product clears the same bound gives the
// same canonical output, so this build fixes the set once.
#pragma once

#include <cstddef>
#include <cstdint>

namespace nc {

constexpr int kMaxPrimes = 48;       // same residue budget as solve.cu:22 kMaxChannels
constexpr int kMaxL = 32;            // limbs of q (solve.cu:1170 accepts L <= 32)
constexpr int kMaxLogN = 16;         // N <= 65536 (the reference stops at 32768, solve.cu:23)
constexpr int kMaxN = 1 << kMaxLogN;
constexpr int kRootLog = kMaxLogN + 1;  // primes are 1 mod 2^17: psi of order 2N for every N <= 2^16

constexpr int kThreads = 256;        // every kernel runs 256-thread CTAs
constexpr int kTile = 256;           // coefficients per decomposition / CRT tile
constexpr int kRowLogMax = 12;       // a row block holds at most 4096 residues (32 KB)
constexpr int kAccExtra = 3;         // CRT accumulator words beyond q's limbs (acc < 2^(bits(q)+69))
constexpr int kBarrettT = 69;        // acc < 2^(bits(q) + kBarrettT)

// Per-prime constants. p = 2^62 - m, m < 2^28 for all primes of the set.
struct PrimeConst {
    uint64_t p;
    uint64_t m;
    uint32_t g;       // floor(2^93 / p): 32-bit reciprocal for the CRT quotient estimate
    uint32_t pad;
};

// Per-(q, N) constants used by the CRT + Barrett stage. Lives in device memory.
struct QConst {
    uint32_t L;          // limbs of q
    uint32_t LW;         // L rounded up to even (accumulator width in the kernels)
    uint32_t k;          // primes used
    uint32_t qbits;      // bit length of q
    uint32_t logN;
    uint32_t pad0;
    uint32_t q[kMaxL + 2];          // q, zero-padded
    uint32_t neg_m[kMaxL + 2];      // (-M) mod q, M = prod of the k primes
    uint32_t mu[4];                 // floor(2^(qbits + kBarrettT + 1) / q), < 2^71
    uint64_t y[kMaxPrimes];         // (M/p_i)^-1 * N^-1 mod p_i
    uint64_t ys[kMaxPrimes];        // Shoup companion of y
    uint32_t mq[kMaxPrimes * (kMaxL + 2)];  // (M/p_i) mod q, row stride kMaxL + 2
};
constexpr int kMqStride = kMaxL + 2;

// One negacyclic product as the kernels see it. All pointers are device pointers.
struct ProductDesc {
    const uint32_t* a;      // N x L limbs (may be null when a_hat is given)
    const uint32_t* b;      // N x L limbs
    uint32_t* c;            // N x L limbs out
    uint64_t* ra;           // k x N residues of a (scratch; holds the product after the row stage)
    uint64_t* rb;           // k x N residues of b (scratch)
    const uint64_t* a_hat;  // optional: a already in the NTT domain (k x N), read instead of a
    uint64_t* hat_out;      // forward-only products write their NTT-domain operand here
    const QConst* qc;
    uint32_t logN;
    uint32_t L;
    uint32_t LW;
    uint32_t k;
    uint32_t mode;          // kModeProduct, kModeCachedA, kModeForward
    uint32_t pad;
};

enum : uint32_t { kModeProduct = 0, kModeCachedA = 1, kModeForward = 2 };

// Geometry of one product: row blocks of N2 = 2^logN2 residues and a column transform of
// N1 = 2^logN1 points over them (N = N1 * N2).
struct Geometry {
    int logN, logN1, logN2;
    int tile;             // coefficients per decomposition / CRT tile
    int tiles;            // tiles per operand
    int rows_per_cta;     // row blocks per row-stage CTA (> 1 only when N2 < 4096)
    int row_ctas;         // CTAs of the row stage
};

inline Geometry geometry(int logN, int k) {
    Geometry g{};
    g.logN = logN;
    g.logN2 = logN < kRowLogMax ? logN : kRowLogMax;
    g.logN1 = logN - g.logN2;
    const int n = 1 << logN;
    g.tile = n < kTile ? n : kTile;
    g.tiles = n / g.tile;
    const int n2 = 1 << g.logN2;
    const int e = n2 >= 16 ? 16 : n2;
    const int threads_per_row = n2 / e;
    g.rows_per_cta = kThreads / threads_per_row;
    const int blocks = k << g.logN1;
    g.row_ctas = (blocks + g.rows_per_cta - 1) / g.rows_per_cta;
    return g;
}

}  // namespace nc
