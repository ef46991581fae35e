// Host-side precompute: the fixed prime set, twiddle tables and per-(q, N) CRT constants.
// This is the planning half of the reference's fherma_init (solve.cu:1150-1487), redone with
// 128-bit integer division instead of bit-serial loops, and for a prime set shared by all N.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "common.h"

namespace nc {

struct HostTables {
    std::vector<PrimeConst> pc;          // kMaxPrimes
    std::vector<uint64_t> psi;           // primitive 2^17-th root of unity per prime
    std::vector<uint64_t> pow32;         // kMaxPrimes * kMaxL
    std::vector<uint64_t> fwd;           // kMaxPrimes * kMaxN * 2 (w, shoup)
    std::vector<uint64_t> inv;           // same for psi^-1
};

// Built once per process (thread-safe); about 100 MB of host memory.
const HostTables& host_tables();

// The primes only (cheap; no twiddles).
const std::vector<PrimeConst>& prime_set();

// Bit length of an L-limb value (0 for zero).
int bit_length(const uint32_t* v, int L);

// Number of primes of the set needed for ring degree 2^logN and a qbits-bit modulus, by the
// reference's bound bitlen(prod p) >= logN + 2 qbits + 4 (solve.cu:1177-1204); -1 if > 48.
// A product of `factors` operands has coefficients below N^(factors-1) q^factors, so its bound is
// (factors - 1) logN + factors qbits + 4 (the reference's bound for factors = 2).
int primes_needed(int logN, int qbits, int factors = 2);

// Fill the CRT + Barrett constants. Returns an empty string or an error message.
std::string build_qconst(const uint32_t* q, int L, int logN, QConst* out, int factors = 2);

// Self-checks run before a plan is handed out, as the reference's fherma_init checks its
// arithmetic before it returns a state (solve.cu:1151-1165, 1285-1314, 1370-1415); unlike its
// L = 28 Barrett check, these hold for every valid q. Each returns "" or what failed.
std::string check_arithmetic();                              // known answers of the host helpers
std::string check_prime_set();                               // primes, their 2^62 - m form, floor(2^93 / p)
std::string check_tables(const HostTables& t, int samples);  // psi, 2^(32 l) mod p, sampled twiddles
std::string check_qconst(const QConst& c);                   // CRT identities and mu of one plan

// ------------------------------------------------------------------ the 30-bit word engine

struct HostTables32 {
    std::vector<PrimeConst32> pc;  // kMaxPrimes32, descending below 2^30
    std::vector<uint32_t> psi;     // primitive 2^17-th root of unity per prime
    std::vector<uint32_t> pow32;   // kMaxPrimes32 * kMaxL: 2^(32 l) mod p
    std::vector<uint32_t> fwd;     // kMaxPrimes32 * kMaxN * 2 (w, floor(w 2^32 / p))
    std::vector<uint32_t> inv;     // same for psi^-1
};

// Built once per process (thread-safe); about 33 MB of host memory.
const HostTables32& host_tables32();
const std::vector<PrimeConst32>& prime_set32();

// Primes of the 30-bit set for the bound of primes_needed (pairs only); -1 if more than 64.
int primes_needed32(int logN, int qbits);

// The 30-bit engine's CRT + Barrett constants. Returns an empty string or an error message.
std::string build_qconst32(const uint32_t* q, int L, int logN, QConst32* out);

std::string check_prime_set32();                                 // primes, 1 mod 2^17, constants
std::string check_tables32(const HostTables32& t, int samples);  // psi, 2^(32 l) mod p, twiddles
std::string check_qconst32(const QConst32& c);                   // CRT identities and mu

// c = a * b mod (X^N + 1, q) by the schoolbook sum on big integers (small N only: the device
// self-test's expected answer).
void schoolbook_negacyclic(int N, int L, const uint32_t* q, const uint32_t* a, const uint32_t* b, uint32_t* c);

// Small helpers shared with the tests of the host math.
uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t p);
uint64_t powmod64(uint64_t a, uint64_t e, uint64_t p);
bool is_prime64(uint64_t n);

}  // namespace nc
