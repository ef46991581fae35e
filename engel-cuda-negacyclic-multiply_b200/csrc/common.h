// Shared constants and plain-old-data structures for the negacyclic product library.
//
// The product c = a*b mod (X^N + 1, q) runs in the residue number system of a fixed set of
// 62-bit primes p = 2^62 - m with p = 1 (mod 2^17), so one prime set and one twiddle table
// serve every ring degree N <= 2^16 and every modulus width. The reference searches primes
// per N (solve.cu:1174-1204); any prime set whose product clears the same bound gives the
// same canonical output, so this build fixes the set once.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#ifdef __CUDACC__
#define NC_HD __host__ __device__
#else
#define NC_HD
#endif

// Tensor-core (tcgen05) instructions exist only in the arch-specific sm_100a target. nvcc
// -arch=sm_100a (the form a CMake project passes) also emits family-portable compute_100 PTX, in
// which the tensor-core kernels compile to empty bodies: a B200 runs the sm_100a code, and
// plan set-up keeps those kernels off any other device. NC_NO_TCGEN05 leaves them out of every
// target (the single-file solve.cu build, whose link-time optimisation cannot take them); the
// residue and CRT stages then run on the integer pipes.
#if defined(NC_NO_TCGEN05)
#define NC_HAS_TCGEN05 0
#elif !defined(__CUDA_ARCH__) || defined(__CUDA_ARCH_FEAT_SM100_ALL) || defined(__CUDA_ARCH_SPECIFIC__) || \
    defined(__CUDA_ARCH_FAMILY_SPECIFIC__)
#define NC_HAS_TCGEN05 1
#else
#define NC_HAS_TCGEN05 0
#endif

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
constexpr int kMaxFactors = 4;       // a chained product multiplies 2 to 4 operands in one pass

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

struct QConst32;

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
    uint32_t logN2;         // row block size of the row configuration (N1 = N >> logN2)
    const uint4* crt_b;     // the plan's byte table for the tensor-core CRT (null: integer-pipe CRT)
    uint32_t factors;       // operands of the product (2: a b; 3, 4: a b x_more[0] [x_more[1]])
    const uint32_t* x_more[kMaxFactors - 2];  // further operands (N x L limbs)
    uint64_t* r_more[kMaxFactors - 2];        // their residues (k x N scratch)
    uint32_t res_tc;        // residue stage of the plain path on the tensor cores (k <= 32)
    // Non-null: the 30-bit word engine runs this product (a pair; k counts its primes, and the
    // residue buffers ra, rb, a_hat and hat_out hold k x N u32).
    const QConst32* qc32;
};

// ------------------------------------------------------------------------------------------
// The 30-bit word engine: primes p < 2^30 with p = 1 (mod 2^17), one u32 residue each.

constexpr int kMaxPrimes32 = 64;         // 4 bytes of v_i x 64 primes = 256, the CRT contraction's K
constexpr int kDecTc32PassPrimes = 32;   // residue MMAs: 4 byte planes x 32 primes = 128 columns

// Per-prime constants of the 30-bit set.
struct PrimeConst32 {
    uint32_t p;
    uint32_t pinv;  // -p^-1 mod 2^32 (Montgomery)
    uint32_t bar;   // floor(2^50 / p): reduction of a 48-bit folded residue sum
    uint32_t quo;   // floor(2^61 / p): the CRT quotient estimate
};

// Per-(q, N) constants of the 30-bit engine's CRT + Barrett stage.
struct QConst32 {
    uint32_t L, LW, k, qbits, logN, pad0;
    uint32_t q[kMaxL + 2];
    uint32_t neg_m[kMaxL + 2];             // (-M) mod q, M = prod of the k primes
    uint32_t mu[4];                        // floor(2^(qbits + kBarrettT + 1) / q)
    uint32_t y[kMaxPrimes32];              // (M/p_i)^-1 N^-1 2^32 mod p_i (2^32: the pointwise Montgomery factor)
    uint32_t ys[kMaxPrimes32];             // floor(y 2^32 / p_i)
    uint32_t mq[kMaxPrimes32 * (kMaxL + 2)];  // (M/p_i) mod q, row stride kMaxL + 2
};

// Operand f of a product (0: a, 1: b, 2..: x_more) and its residue buffer.
NC_HD inline const uint32_t* factor_limbs(const ProductDesc& d, int f) {
    return f == 0 ? d.a : f == 1 ? d.b : d.x_more[f - 2];
}
NC_HD inline uint64_t* factor_residues(const ProductDesc& d, int f) {
    return f == 0 ? d.ra : f == 1 ? d.rb : d.r_more[f - 2];
}

enum : uint32_t { kModeProduct = 0, kModeCachedA = 1, kModeForward = 2 };

// Device-wide twiddle tables (built once per device). Entry j of prime i sits at
// fwd[i * kMaxN + j] = psi^bitrev16(j) with its Shoup companion (inv: psi^-bitrev16(j)); the
// first N entries are the merged twiddles of every ring degree N <= 2^16.
struct Tables {
    const ulonglong2* fwd;    // [kMaxPrimes][kMaxN]
    const ulonglong2* inv;    // [kMaxPrimes][kMaxN]
    const uint64_t* pow32;    // [kMaxPrimes][kMaxL]: 2^(32 l) mod p_i
    const uint64_t* primes;   // [kMaxPrimes]
    const uint4* res_w;       // [kMaxPrimes][8 K chunks][8 byte planes][16 B]: byte c of 2^(8 b) mod p_i
    // 30-bit engine
    const uint2* fwd32;           // [kMaxPrimes32][kMaxN]: psi^bitrev16(j) and floor(w 2^32 / p)
    const uint2* inv32;           // [kMaxPrimes32][kMaxN]: psi^-bitrev16(j) and its companion
    const PrimeConst32* pc32;     // [kMaxPrimes32]
    const uint32_t* pow32_32;     // [kMaxPrimes32][kMaxL]: 2^(32 l) mod p_i
    const uint4* res_w32;         // [prime pairs][8 K chunks][8 rows: 4 byte planes of each][16 B]
};

// Dynamic shared memory of each stage.
NC_HD constexpr size_t smax(size_t a, size_t b) { return a > b ? a : b; }
// residue stage: limb tile overlaid by the residues, then 2^(32 l) mod p_i and p_i for k primes
NC_HD constexpr size_t dec_main_bytes(int k) { return smax(size_t(kTile) * kMaxL * 4, size_t(kTile) * 8 * size_t(k)); }
NC_HD constexpr size_t dec_smem_bytes(int k) { return dec_main_bytes(k) + size_t(k) * (kMaxL + 1) * 8; }
NC_HD constexpr size_t row_smem_bytes(int threads, int logE) { return size_t(2) * size_t(threads) * (size_t(1) << logE) * 8; }
NC_HD constexpr size_t crt_smem_bytes(int k) {
    return smax(size_t(kTile) * 8 * size_t(k), size_t(kTile) * kMaxL * 4)  // residues / output staging
           + size_t(k) * kMqStride * 4                                       // M/p_i mod q
           + size_t(k) * 8 * 3                                               // y, y shoup, p
           + size_t(kMqStride) * 4 * 2 + 16;                                 // -M mod q, q, mu
}

// Tensor-core CRT (plain path): a 256-coefficient tile is two 128-row halves of A, each 128 rows x
// 256 K bytes (8 bytes of v_i per prime, so at most 32 primes); the plan's table B has NC output
// byte columns (4 LW + 7 rounded up to 16) x 256 K bytes.
constexpr int kCrtTcMaxPrimes = 32;
constexpr int kCrtTcHalfBytes = 128 * 256;
NC_HD constexpr int crt_tc_cols(int LW) { return (4 * LW + 7 + 15) / 16 * 16; }
NC_HD constexpr size_t crt_tc_table_bytes(int LW) { return size_t(crt_tc_cols(LW)) * 256; }
// tensor-memory columns of one tile: two accumulators of NC columns, rounded up to 256 or 512
NC_HD constexpr uint32_t crt_tc_tmem_cols(int LW) { return 2 * crt_tc_cols(LW) <= 256 ? 256u : 512u; }
// Operands and constants; raised so that no more CTAs share an SM
// than its 512 tensor-memory columns hold (two accumulators of NC columns, rounded up to 256 or 512).
NC_HD constexpr size_t crt_tc_smem_bytes(int LW) {
    return smax(size_t(2) * kCrtTcHalfBytes + crt_tc_table_bytes(LW) + size_t(kCrtTcMaxPrimes) * 8 * 3 +
                    size_t(kMqStride) * 4 * 2 + 16 + 16,
                (size_t(233472) / (512 / crt_tc_tmem_cols(LW) + 1) + 16) / 16 * 16);
}

// Residue stage on the tensor cores (plain path): a tile of 128 coefficients (the MMA's M) x 128
// K bytes of limbs, the weight bytes of the k primes (1 KB each), and p_i; the primes go through
// the MMA in passes of 16 (128 accumulator columns), so tensor memory holds four CTAs per SM. The
// shared memory is raised to keep it at four.
constexpr int kDecTcRows = 128;
constexpr int kDecTcPassPrimes = 16;
constexpr uint32_t kDecTcCols = 128;
NC_HD constexpr size_t dec_tc_smem_bytes(int k) {
    return smax(size_t(kDecTcRows) * 128 + size_t((k + 1) & ~1) * 1024 + size_t(kMaxPrimes) * 8,
                (size_t(233472) / (512 / kDecTcCols + 1) + 16) / 16 * 16);
}

// How the row stage tiles a product: row blocks of N2 = 2^logN2 residues, each thread holding
// 2^logE of them per register pass (the NTT radix), CTAs of `threads` threads. The column
// transform then has N1 = N / N2 points (at most 32).
struct RowConfig {
    int logN2;
    int logE;
    int threads;
};

constexpr int kMaxLogN1 = 5;
constexpr int kRowLogCap = 13;

inline RowConfig default_row_config(int logN) {
    RowConfig c{};
    c.logN2 = logN < kRowLogMax ? logN : kRowLogMax;
    c.logE = 4;
    c.threads = 256;
    return c;
}

// Geometry of one product under a row configuration.
struct Geometry {
    int logN, logN1, logN2, logE, row_threads;
    int tile;             // coefficients per decomposition / CRT tile
    int tiles;            // tiles per operand
    int rows_per_cta;     // row blocks per row-stage CTA
    int row_ctas;         // CTAs of the row stage
};

inline bool row_config_valid(int logN, const RowConfig& c) {
    if (c.logN2 < 1 || c.logN2 > kRowLogCap || c.logN2 > logN) return false;
    if (logN - c.logN2 > kMaxLogN1) return false;
    if (logN > kRowLogMax && c.logN2 < logN - kMaxLogN1) return false;
    if (c.logE != 3 && c.logE != 4) return false;
    if (c.threads != 256 && c.threads != 512) return false;
    const int le = c.logE < c.logN2 ? c.logE : c.logN2;
    const int t = 1 << (c.logN2 - le);
    return t <= c.threads;
}

inline Geometry geometry(int logN, int k, const RowConfig& c) {
    Geometry g{};
    g.logN = logN;
    g.logN2 = c.logN2;
    g.logN1 = logN - c.logN2;
    g.logE = c.logE;
    g.row_threads = c.threads;
    const int n = 1 << logN;
    g.tile = n < kTile ? n : kTile;
    g.tiles = n / g.tile;
    const int le = c.logE < c.logN2 ? c.logE : c.logN2;
    const int threads_per_row = 1 << (c.logN2 - le);
    g.rows_per_cta = c.threads / threads_per_row;
    const int blocks = k << g.logN1;
    g.row_ctas = (blocks + g.rows_per_cta - 1) / g.rows_per_cta;
    return g;
}

}  // namespace nc
