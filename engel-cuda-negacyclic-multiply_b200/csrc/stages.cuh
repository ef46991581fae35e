// The three stages of one negacyclic product, written as CTA-level device functions so the
// plain per-call kernels and the persistent batched kernel share them.
//
//   stage 1  residues   limbs -> residues mod each prime (solve.cu:533-570 computes the same
//                       residues) and the first log2(N1) forward NTT stages over columns
//   stage 2  row blocks per (prime, row block of N2 residues): forward NTT of a and of b,
//                       pointwise product, inverse NTT (solve.cu:952-1044, 620-628)
//   stage 3  CRT        last log2(N1) inverse stages over columns, then CRT and Barrett
//                       reduction mod q into L limbs (solve.cu:630-642, 752-836)
//
// The NTT is the merged negacyclic form: forward Cooley-Tukey with twiddles psi^bitrev(j)
// (natural order in, bit-reversed order out) and inverse Gentleman-Sande with psi^-bitrev(j)
// (bit-reversed in, natural out), so no twist, untwist or bit-reversal pass exists. N^-1 is
// folded into the CRT constant y_i. Residue rows are k x N u64, prime-major.
//
// This header defines static __constant__ data: every translation unit that includes it has its
// own copy and uploads it with upload_prime_constants() before its first launch.
#pragma once

#include <cstdint>

#include "arith.cuh"
#include "common.h"

namespace nc {

// Per-prime constants, read with warp-uniform indices.
static __constant__ PrimeConst c_pc[kMaxPrimes];
static __constant__ uint64_t c_pow32[kMaxPrimes * kMaxL];  // 2^(32 l) mod p_i

static inline cudaError_t upload_prime_constants(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = cudaMemcpyToSymbol(c_pc, pc, sizeof(PrimeConst) * kMaxPrimes);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_pow32, pow32, sizeof(uint64_t) * kMaxPrimes * kMaxL);
    return e;
}

#define NC_LW_CASES(X) X(2) X(4) X(6) X(8) X(10) X(12) X(14) X(16) X(18) X(20) X(22) X(24) X(26) X(28) X(30) X(32)

// ------------------------------------------------------------------------------------------
// stage 1: residues + forward column stages

// Loads the CTA's tile (N1 segments of C consecutive coefficients) into shared memory. When
// every segment starts on 16 bytes, one pass over all segments' 16-byte chunks keeps every
// thread busy (a pass per segment left most of them idle for short segments).
__device__ __forceinline__ void load_tile(const uint32_t* x, int N2, int L, int j0, int C, int N1,
                                          uint32_t* s_in) {
    const int seg = C * L;
    if (((size_t(N2) * L | size_t(j0) * L | size_t(seg)) & 3) == 0) {
        const int seg4 = seg >> 2;
        for (int w = threadIdx.x; w < N1 * seg4; w += blockDim.x) {
            const int u = w / seg4, c = w - u * seg4;
            reinterpret_cast<uint4*>(s_in + u * seg)[c] =
                __ldg(reinterpret_cast<const uint4*>(x + (size_t(u) * N2 + j0) * L) + c);
        }
        return;
    }
    for (int u = 0; u < N1; ++u) {
        const uint32_t* src = x + (size_t(u) * N2 + j0) * L;
        uint32_t* dst = s_in + u * seg;
        for (int w = threadIdx.x; w < seg; w += blockDim.x) dst[w] = __ldg(src + w);
    }
}

// The CTA's staged output tile (N1 segments of C coefficients in s_out) to its place in c.
__device__ __forceinline__ void store_tile(uint32_t* c, int N2, int L, int j0, int C, int N1, const uint32_t* s_out) {
    const int seg = C * L;
    if (((size_t(N2) * L | size_t(j0) * L | size_t(seg)) & 3) == 0) {
        const int seg4 = seg >> 2;
        for (int w = threadIdx.x; w < N1 * seg4; w += blockDim.x) {
            const int u = w / seg4, x = w - u * seg4;
            reinterpret_cast<uint4*>(c + (size_t(u) * N2 + j0) * L)[x] = reinterpret_cast<const uint4*>(s_out + u * seg)[x];
        }
        return;
    }
    for (int u = 0; u < N1; ++u) {
        uint32_t* dst = c + (size_t(u) * N2 + j0) * L;
        const uint32_t* src = s_out + u * seg;
        for (int w = threadIdx.x; w < seg; w += blockDim.x) dst[w] = src[w];
    }
}

// Thread t owns coefficient t of the tile: its limbs stay in registers while it walks the
// primes two at a time (two independent carry chains), writing residues in [0, 2p) to
// s_res[i * T + t]. s_res overlays the limb tile, so the limbs are read first. The weights
// 2^(32 l) mod p_i come from shared memory (s_pow, row stride kMaxL): every lane reads the same
// word, one broadcast per warp, which keeps them off the constant-load path.
template <int LW>
__device__ __forceinline__ void dec_residues(const uint32_t* s_in, int L, int k, int T, const uint64_t* s_pow,
                                             uint64_t* s_res) {
    const int t = threadIdx.x;
    const bool active = t < T;
    uint32_t x[LW];
#pragma unroll
    for (int l = 0; l < LW; ++l) x[l] = 0;
    if (active) {
        const uint32_t* src = s_in + t * L;
        if ((L & 3) == 0) {
#pragma unroll
            for (int l = 0; l < LW; l += 4)
                if (l < L) {
                    const uint4 v = *reinterpret_cast<const uint4*>(src + l);
                    x[l] = v.x;
                    x[l + 1] = v.y;
                    x[l + 2] = v.z;
                    x[l + 3] = v.w;
                }
        } else if ((L & 1) == 0) {
#pragma unroll
            for (int l = 0; l < LW; l += 2)
                if (l < L) {
                    const uint2 v = *reinterpret_cast<const uint2*>(src + l);
                    x[l] = v.x;
                    x[l + 1] = v.y;
                }
        } else {
#pragma unroll
            for (int l = 0; l < LW; ++l)
                if (l < L) x[l] = src[l];
        }
    }
    __syncthreads();  // the limb tile is in registers; s_res may now overwrite it
    if (!active) return;
#pragma unroll 1
    for (int i = 0; i < k; i += 2) {
        const int i2 = (i + 1 < k) ? i + 1 : i;
        const uint64_t* c1 = s_pow + i * kMaxL;
        const uint64_t* c2 = s_pow + i2 * kMaxL;
        uint32_t a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
        uint32_t e0 = 0, e1 = 0, e2 = 0, f0 = 0, f1 = 0, f2 = 0;
#pragma unroll
        for (int l = 0; l < LW; ++l) {
            const uint64_t c = c1[l], dd = c2[l];
            mac_u32x64(x[l], uint32_t(c), uint32_t(c >> 32), a0, a1, a2, b0, b1, b2);
            mac_u32x64(x[l], uint32_t(dd), uint32_t(dd >> 32), e0, e1, e2, f0, f1, f2);
        }
        s_res[size_t(i) * T + t] = reduce_limb_sum(a0, a1, a2, b0, b1, b2, c_pc[i].m);
        if (i + 1 < k) s_res[size_t(i2) * T + t] = reduce_limb_sum(e0, e1, e2, f0, f1, f2, c_pc[i2].m);
    }
}

// Forward column stages (global stages m = 1 .. N1/2) of one column held in registers.
template <int LOG_N1>
__device__ __forceinline__ void column_forward(const ulonglong2* tw, uint64_t p, uint64_t (&v)[1 << LOG_N1]) {
    constexpr int N1 = 1 << LOG_N1;
    const uint64_t p2 = 2 * p;
#pragma unroll
    for (int s = 0; s < LOG_N1; ++s) {
        const int half = N1 >> (s + 1);
#pragma unroll
        for (int blk = 0; blk < (1 << s); ++blk) {
            const ulonglong2 w = __ldg(tw + (1 << s) + blk);
#pragma unroll
            for (int jj = 0; jj < half; ++jj) {
                const int u = blk * 2 * half + jj;
                ct_bfly(v[u], v[u + half], w.x, w.y, p, p2);
            }
        }
    }
}

// The same stages on one half-subtree of a longer column: the 2^LOG_N1 values under node `root`
// of the merged twiddle tree (the full column is root 1), whose stage s uses twiddle
// (root << s) + block.
template <int LOG_N1>
__device__ __forceinline__ void column_forward_root(const ulonglong2* tw, int root, uint64_t p,
                                                    uint64_t (&v)[1 << LOG_N1]) {
    constexpr int N1 = 1 << LOG_N1;
    const uint64_t p2 = 2 * p;
#pragma unroll
    for (int s = 0; s < LOG_N1; ++s) {
        const int half = N1 >> (s + 1);
#pragma unroll
        for (int blk = 0; blk < (1 << s); ++blk) {
            const ulonglong2 w = __ldg(tw + (root << s) + blk);
#pragma unroll
            for (int jj = 0; jj < half; ++jj) {
                const int u = blk * 2 * half + jj;
                ct_bfly(v[u], v[u + half], w.x, w.y, p, p2);
            }
        }
    }
}

// Inverse column stages (global stages m = N1/2 .. 1) of one column held in registers.
template <int LOG_N1>
__device__ __forceinline__ void column_inverse(const ulonglong2* tw, uint64_t p, uint64_t (&v)[1 << LOG_N1]) {
    constexpr int N1 = 1 << LOG_N1;
    const uint64_t p2 = 2 * p;
#pragma unroll
    for (int s = LOG_N1 - 1; s >= 0; --s) {
        const int half = N1 >> (s + 1);
#pragma unroll
        for (int blk = 0; blk < (1 << s); ++blk) {
            const ulonglong2 w = __ldg(tw + (1 << s) + blk);
#pragma unroll
            for (int jj = 0; jj < half; ++jj) {
                const int u = blk * 2 * half + jj;
                gs_bfly(v[u], v[u + half], w.x, w.y, p, p2);
            }
        }
    }
}

// Inverse stages of one half-subtree of a longer column (root as in column_forward_root).
template <int LOG_N1>
__device__ __forceinline__ void column_inverse_root(const ulonglong2* tw, int root, uint64_t p,
                                                    uint64_t (&v)[1 << LOG_N1]) {
    constexpr int N1 = 1 << LOG_N1;
    const uint64_t p2 = 2 * p;
#pragma unroll
    for (int s = LOG_N1 - 1; s >= 0; --s) {
        const int half = N1 >> (s + 1);
#pragma unroll
        for (int blk = 0; blk < (1 << s); ++blk) {
            const ulonglong2 w = __ldg(tw + (root << s) + blk);
#pragma unroll
            for (int jj = 0; jj < half; ++jj) {
                const int u = blk * 2 * half + jj;
                gs_bfly(v[u], v[u + half], w.x, w.y, p, p2);
            }
        }
    }
}

// A u64 from the neighbouring lane (lane ^ 1) of a full warp.
__device__ __forceinline__ uint64_t shfl_pair(uint64_t x) {
    return (uint64_t(__shfl_xor_sync(0xffffffffu, uint32_t(x >> 32), 1)) << 32) |
           __shfl_xor_sync(0xffffffffu, uint32_t(x), 1);
}

// Items (prime i, column j) of the tile: column transform from s_res, store the residue rows.
// A warp may span two primes, so p_i comes from shared memory (s_p) rather than constant memory.
template <int LOG_N1>
__device__ void dec_columns(const Tables& t, int k, int N, int T, int j0, const uint64_t* s_res, const uint64_t* s_p,
                            uint64_t* R) {
    constexpr int N1 = 1 << LOG_N1;
    const int C = T >> LOG_N1;
    const int N2 = N >> LOG_N1;
    for (int w = threadIdx.x; w < k * C; w += blockDim.x) {
        const int i = w / C, j = w - i * C;
        uint64_t v[N1];
#pragma unroll
        for (int u = 0; u < N1; ++u) v[u] = s_res[size_t(i) * T + u * C + j];
        if (LOG_N1 > 0) column_forward<LOG_N1>(t.fwd + size_t(i) * kMaxN, s_p[i], v);
        uint64_t* row = R + size_t(i) * N + j0 + j;
#pragma unroll
        for (int u = 0; u < N1; ++u) __stcg(row + size_t(u) * N2, v[u]);
    }
}

template <int LW>
__device__ void dec_tile(const ProductDesc& d, const Tables& t, int operand, int tile, uint8_t* smem) {
    const int N = 1 << d.logN;
    const int logN1 = int(d.logN) - int(d.logN2);
    const int T = N < kTile ? N : kTile;
    const int C = T >> logN1;
    const int L = int(d.L), k = int(d.k);
    const uint32_t* x = factor_limbs(d, operand);
    uint64_t* R = factor_residues(d, operand);
    uint32_t* s_in = reinterpret_cast<uint32_t*>(smem);
    uint64_t* s_res = reinterpret_cast<uint64_t*>(smem);
    uint64_t* s_pow = reinterpret_cast<uint64_t*>(smem + dec_main_bytes(k));
    uint64_t* s_p = s_pow + size_t(k) * kMaxL;
    const int j0 = tile * C;

    __syncthreads();  // the previous user of shared memory (persistent CTAs) is done
    for (int w = threadIdx.x; w < k * kMaxL; w += blockDim.x) s_pow[w] = __ldg(t.pow32 + w);
    for (int w = threadIdx.x; w < k; w += blockDim.x) s_p[w] = __ldg(t.primes + w);
    pdl_wait();  // the operand and the residue rows belong to the stream's previous kernels
    load_tile(x, N >> logN1, L, j0, C, 1 << logN1, s_in);
    __syncthreads();
    dec_residues<LW>(s_in, L, k, T, s_pow, s_res);
    __syncthreads();
    switch (logN1) {
        case 0: dec_columns<0>(t, k, N, T, j0, s_res, s_p, R); break;
        case 1: dec_columns<1>(t, k, N, T, j0, s_res, s_p, R); break;
        case 2: dec_columns<2>(t, k, N, T, j0, s_res, s_p, R); break;
        case 3: dec_columns<3>(t, k, N, T, j0, s_res, s_p, R); break;
        case 4: dec_columns<4>(t, k, N, T, j0, s_res, s_p, R); break;
        default: dec_columns<5>(t, k, N, T, j0, s_res, s_p, R); break;
    }
}

// ------------------------------------------------------------------------------------------
// stage 2: row blocks

// 16-byte-chunk XOR swizzle inside 128-byte rows of a u64 buffer.
__device__ __forceinline__ int swz(int x) {
    const int c = x >> 1;
    const int pc = (c & ~7) | ((c ^ (c >> 3)) & 7);
    return (pc << 1) | (x & 1);
}

template <int LOG_N2_, int LOG_E>
struct RowShape {
    static constexpr int LOG_N2 = LOG_N2_;
    static constexpr int N2 = 1 << LOG_N2;
    static constexpr int LE = LOG_N2 < LOG_E ? LOG_N2 : LOG_E;
    static constexpr int E = 1 << LE;
    static constexpr int T = N2 / E;  // threads per row block
    static constexpr int NPASS = (LOG_N2 + LE - 1) / LE;
    __host__ __device__ static constexpr int l0(int pass) { return pass * LE; }
    __host__ __device__ static constexpr int r(int pass) {
        return (LOG_N2 - pass * LE) < LE ? (LOG_N2 - pass * LE) : LE;
    }
    __host__ __device__ static constexpr int lolog(int pass) { return LOG_N2 - l0(pass) - r(pass); }
};

// Element index (inside the row block) of register slot e in pass PASS for thread lt.
// A pass runs r stages on groups of 2^r elements x = hi * (N2 >> l0) + s * 2^lolog + lo.
template <class S, int PASS>
__device__ __forceinline__ int row_index(int lt, int e) {
    constexpr int R = S::r(PASS), LL = S::lolog(PASS);
    const int q = e >> R, s = e & ((1 << R) - 1);
    const int g = lt + S::T * q;
    const int hi = g >> LL, lo = g & ((1 << LL) - 1);
    return (hi << (S::LOG_N2 - S::l0(PASS))) + (s << LL) + lo;
}

template <class S, int PASS, bool FWD>
__device__ __forceinline__ void row_pass(uint64_t (&v)[S::E], const ulonglong2* tw, int base, int lt, uint64_t p) {
    constexpr int R = S::r(PASS), LL = S::lolog(PASS), L0 = S::l0(PASS);
    const uint64_t p2 = 2 * p;
#pragma unroll
    for (int q = 0; q < (S::E >> R); ++q) {
        const int g = lt + S::T * q;
        const int hi = g >> LL;
#pragma unroll
        for (int jj = 0; jj < R; ++jj) {
            const int j = FWD ? jj : R - 1 - jj;
            const int half = 1 << (R - 1 - j);
            // twiddle of local stage l = L0 + j, block b: (N1 + u) 2^l + hi 2^j + (s >> (R - j))
            const int twbase = (base << (L0 + j)) + (hi << j);
#pragma unroll
            for (int blk = 0; blk < (1 << j); ++blk) {
                const ulonglong2 w = __ldg(tw + twbase + blk);
#pragma unroll
                for (int s0 = 0; s0 < half; ++s0) {
                    const int e = q * (1 << R) + blk * 2 * half + s0;
                    if (FWD)
                        ct_bfly(v[e], v[e + half], w.x, w.y, p, p2);
                    else
                        gs_bfly(v[e], v[e + half], w.x, w.y, p, p2);
                }
            }
        }
    }
}

template <class S, int PASS>
__device__ __forceinline__ void row_store(const uint64_t (&v)[S::E], uint64_t* buf, int lt) {
    if (S::lolog(PASS) == 0 && S::r(PASS) >= 1) {
#pragma unroll
        for (int e = 0; e < S::E; e += 2) {
            const int x = row_index<S, PASS>(lt, e);
            reinterpret_cast<ulonglong2*>(buf)[swz(x) >> 1] = make_ulonglong2(v[e], v[e + 1]);
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) buf[swz(row_index<S, PASS>(lt, e))] = v[e];
    }
}

template <class S, int PASS>
__device__ __forceinline__ void row_load(uint64_t (&v)[S::E], const uint64_t* buf, int lt) {
    if (S::lolog(PASS) == 0 && S::r(PASS) >= 1) {
#pragma unroll
        for (int e = 0; e < S::E; e += 2) {
            const int x = row_index<S, PASS>(lt, e);
            const ulonglong2 pr = reinterpret_cast<const ulonglong2*>(buf)[swz(x) >> 1];
            v[e] = pr.x;
            v[e + 1] = pr.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = buf[swz(row_index<S, PASS>(lt, e))];
    }
}

// Forward passes PASS..NPASS-1 from registers in pass-PASS layout; ends in last-pass layout.
template <class S, int PASS>
__device__ __forceinline__ void row_forward_from(uint64_t (&v)[S::E], uint64_t* buf, const ulonglong2* tw,
                                                 int base, int lt, uint64_t p) {
    row_pass<S, PASS, true>(v, tw, base, lt, p);
    if constexpr (PASS + 1 < S::NPASS) {
        __syncthreads();
        row_store<S, PASS>(v, buf, lt);
        __syncthreads();
        row_load<S, PASS + 1>(v, buf, lt);
        row_forward_from<S, PASS + 1>(v, buf, tw, base, lt, p);
    }
}

// Inverse passes PASS..0 from registers in pass-PASS layout; ends in pass-0 layout.
template <class S, int PASS>
__device__ __forceinline__ void row_inverse_from(uint64_t (&v)[S::E], uint64_t* buf, const ulonglong2* tw,
                                                 int base, int lt, uint64_t p) {
    row_pass<S, PASS, false>(v, tw, base, lt, p);
    if constexpr (PASS > 0) {
        __syncthreads();
        row_store<S, PASS>(v, buf, lt);
        __syncthreads();
        row_load<S, PASS - 1>(v, buf, lt);
        row_inverse_from<S, PASS - 1>(v, buf, tw, base, lt, p);
    }
}

// One CTA of THREADS threads handles ROWS = THREADS / T row blocks: block rb = item * ROWS +
// (tid / T) is prime rb >> logN1, row u = rb & (N1 - 1), residues [u N2, (u + 1) N2).
template <int LOG_N2, int LOG_E, int THREADS>
__device__ void row_blocks(const ProductDesc& d, const Tables& t, int item, uint8_t* smem) {
    using S = RowShape<LOG_N2, LOG_E>;
    static_assert(S::T <= THREADS, "row block needs more threads than the CTA has");
    constexpr int ROWS = THREADS / S::T;
    constexpr int LAST = S::NPASS - 1;
    const int logN1 = int(d.logN) - LOG_N2;
    const int N = 1 << d.logN;
    const int rr = threadIdx.x / S::T, lt = threadIdx.x - rr * S::T;
    const int rb = item * ROWS + rr;
    const bool active = rb < (int(d.k) << logN1);
    const int i = active ? rb >> logN1 : 0;
    const int u = rb & ((1 << logN1) - 1);
    const uint64_t p = c_pc[i].p, m = c_pc[i].m;
    const int base = (1 << logN1) + u;
    const size_t off = size_t(i) * N + size_t(u) * S::N2;
    uint64_t* buf = reinterpret_cast<uint64_t*>(smem) + rr * S::N2;
    uint64_t* buf_a = reinterpret_cast<uint64_t*>(smem) + size_t(ROWS) * S::N2 + rr * S::N2;
    const ulonglong2* twf = t.fwd + size_t(i) * kMaxN;
    const ulonglong2* twi = t.inv + size_t(i) * kMaxN;
    uint64_t v[S::E];

    __syncthreads();  // shared memory of a previous item is free
    pdl_wait();       // the residues come from the stream's previous kernel
    if (d.mode == kModeCachedA) {
        // a is already in the NTT domain: stage it into buf_a
#pragma unroll
        for (int e = 0; e < S::E; ++e) {
            const int x = row_index<S, 0>(lt, e);
            buf_a[swz(x)] = active ? __ldcg(d.a_hat + off + x) : 0;
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = active ? __ldcg(d.ra + off + row_index<S, 0>(lt, e)) : 0;
        row_forward_from<S, 0>(v, buf, twf, base, lt, p);
        if (d.mode == kModeForward) {
            __syncthreads();
            row_store<S, LAST>(v, buf, lt);
            __syncthreads();
            row_load<S, 0>(v, buf, lt);
            if (active) {
#pragma unroll
                for (int e = 0; e < S::E; ++e) __stcg(d.hat_out + off + row_index<S, 0>(lt, e), v[e]);
            }
            return;
        }
        row_store<S, LAST>(v, buf_a, lt);
    }
    // factors 1 .. factors-1: forward transform, then pointwise product with the running product
    // in buf_a (each thread reads and writes only its own positions there)
    const int nf = d.mode == kModeProduct ? int(d.factors) : 2;
    for (int f = 1; f < nf; ++f) {
        if (f > 1) row_store<S, LAST>(v, buf_a, lt);
        const uint64_t* R = factor_residues(d, f);
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = active ? __ldcg(R + off + row_index<S, 0>(lt, e)) : 0;
        row_forward_from<S, 0>(v, buf, twf, base, lt, p);
        __syncthreads();
        const uint64_t p2 = 2 * p;
        if (S::lolog(LAST) == 0 && S::r(LAST) >= 1) {
#pragma unroll
            for (int e = 0; e < S::E; e += 2) {
                const int x = row_index<S, LAST>(lt, e);
                const ulonglong2 pr = reinterpret_cast<const ulonglong2*>(buf_a)[swz(x) >> 1];
                v[e] = mulmod_special(csub(csub(pr.x, p2), p), v[e], m);
                v[e + 1] = mulmod_special(csub(csub(pr.y, p2), p), v[e + 1], m);
            }
        } else {
#pragma unroll
            for (int e = 0; e < S::E; ++e) {
                const uint64_t av = buf_a[swz(row_index<S, LAST>(lt, e))];
                v[e] = mulmod_special(csub(csub(av, p2), p), v[e], m);
            }
        }
    }
    row_inverse_from<S, LAST>(v, buf, twi, base, lt, p);
    if (active) {
#pragma unroll
        for (int e = 0; e < S::E; ++e) __stcg(d.ra + off + row_index<S, 0>(lt, e), v[e]);
    }
}

// ------------------------------------------------------------------------------------------
// stage 3: inverse column stages + CRT + Barrett

template <int LOG_N1>
__device__ void crt_columns(const ProductDesc& d, const Tables& t, int tile, const uint64_t* s_p, uint64_t* s_res) {
    constexpr int N1 = 1 << LOG_N1;
    const int N = 1 << d.logN;
    const int N2 = N >> LOG_N1;
    const int T = N < kTile ? N : kTile;
    const int C = T >> LOG_N1;
    const int k = int(d.k);
    const int j0 = tile * C;
    for (int w = threadIdx.x; w < k * C; w += blockDim.x) {
        const int i = w / C, j = w - i * C;
        const uint64_t* row = d.ra + size_t(i) * N + j0 + j;
        uint64_t v[N1];
#pragma unroll
        for (int u = 0; u < N1; ++u) v[u] = __ldcg(row + size_t(u) * N2);
        if (LOG_N1 > 0) column_inverse<LOG_N1>(t.inv + size_t(i) * kMaxN, s_p[i], v);
#pragma unroll
        for (int u = 0; u < N1; ++u) s_res[size_t(i) * T + u * C + j] = v[u];
    }
}

// acc[OFF..W) += lo(v * M[l]) placed at word OFF + l  (one carry chain; top word takes the carry)
template <int LW, int OFF, int W>
__device__ __forceinline__ void mac_lo(uint32_t (&acc)[W], const uint32_t* M, uint32_t v) {
    asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF]) : "r"(v), "r"(M[0]));
#pragma unroll
    for (int l = 1; l < LW; ++l) asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF + l]) : "r"(v), "r"(M[l]));
#pragma unroll
    for (int w = OFF + LW; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, 0;" : "+r"(acc[w]));
    asm volatile("addc.u32 %0, %0, 0;" : "+r"(acc[W - 1]));
}

// acc[OFF..W) += hi(v * M[l]) placed at word OFF + l
template <int LW, int OFF, int W>
__device__ __forceinline__ void mac_hi(uint32_t (&acc)[W], const uint32_t* M, uint32_t v) {
    asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF]) : "r"(v), "r"(M[0]));
#pragma unroll
    for (int l = 1; l < LW; ++l) asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF + l]) : "r"(v), "r"(M[l]));
#pragma unroll
    for (int w = OFF + LW; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, 0;" : "+r"(acc[w]));
    if (OFF + LW < W) asm volatile("addc.u32 %0, %0, 0;" : "+r"(acc[W - 1]));
}

__device__ __forceinline__ uint32_t funnel(uint32_t lo, uint32_t hi, int sh) { return __funnelshift_r(lo, hi, sh); }

// r (LW + 1 words) := acc mod q, for acc < 2^(qbits + kBarrettT).
template <int LW, int W>
__device__ __forceinline__ void barrett(const uint32_t (&acc)[W], const uint32_t* q, const uint32_t* mu, int qbits,
                                        uint32_t (&r)[LW + 1]) {
    // y = floor(acc / 2^(qbits-1)): 3 words. qbits - 1 lies in [32 (L-1), 32 L), L in {LW-1, LW}.
    const int b1 = qbits - 1;
    const int sh = b1 & 31;
    uint32_t y0, y1, y2;
    if ((b1 >> 5) == LW - 1) {
        y0 = funnel(acc[LW - 1], acc[LW], sh);
        y1 = funnel(acc[LW], acc[LW + 1], sh);
        y2 = funnel(acc[LW + 1], acc[LW + 2], sh);
    } else {
        y0 = funnel(acc[LW - 2], acc[LW - 1], sh);
        y1 = funnel(acc[LW - 1], acc[LW], sh);
        y2 = funnel(acc[LW], acc[LW + 1], sh);
    }
    // t = y * mu (6 words), qh = t >> (kBarrettT + 2) = t >> 71
    uint32_t tt[6] = {0, 0, 0, 0, 0, 0};
    {
        const uint32_t ys[3] = {y0, y1, y2};
        const uint32_t ms[3] = {mu[0], mu[1], mu[2]};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            uint64_t carry = 0;
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) {
                const uint64_t cur = uint64_t(tt[a + bb]) + uint64_t(ys[a]) * ms[bb] + carry;
                tt[a + bb] = uint32_t(cur);
                carry = cur >> 32;
            }
            tt[a + 3] = uint32_t(carry);
        }
    }
    const uint32_t qs[3] = {funnel(tt[2], tt[3], 7), funnel(tt[3], tt[4], 7), funnel(tt[4], tt[5], 7)};
    // prod = qh * q, low LW + 1 words
    uint32_t prod[LW + 1];
#pragma unroll
    for (int w = 0; w <= LW; ++w) prod[w] = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        uint64_t carry = 0;
#pragma unroll
        for (int l = 0; l + a <= LW; ++l) {
            const uint32_t ql = l < LW ? q[l] : 0u;
            const uint64_t cur = uint64_t(prod[l + a]) + uint64_t(qs[a]) * ql + carry;
            prod[l + a] = uint32_t(cur);
            carry = cur >> 32;
        }
    }
    // r = acc - prod (mod 2^(32 (LW + 1)))
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r[0]) : "r"(acc[0]), "r"(prod[0]));
#pragma unroll
    for (int w = 1; w < LW; ++w) asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r[w]) : "r"(acc[w]), "r"(prod[w]));
    asm volatile("subc.u32 %0, %1, %2;" : "=r"(r[LW]) : "r"(acc[LW]), "r"(prod[LW]));
    // at most two subtractions of q
#pragma unroll
    for (int fix = 0; fix < 2; ++fix) {
        uint32_t s[LW + 1];
        uint32_t borrow;
        asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(s[0]) : "r"(r[0]), "r"(q[0]));
#pragma unroll
        for (int w = 1; w < LW; ++w) asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(s[w]) : "r"(r[w]), "r"(q[w]));
        asm volatile("subc.cc.u32 %0, %1, 0;" : "=r"(s[LW]) : "r"(r[LW]));
        asm volatile("subc.u32 %0, 0, 0;" : "=r"(borrow));
        const bool keep = borrow != 0;  // r < q
#pragma unroll
        for (int w = 0; w <= LW; ++w) r[w] = keep ? r[w] : s[w];
    }
}

template <int LW>
__device__ void crt_coeffs(const ProductDesc& d, const Tables& t, int tile, uint8_t* smem) {
    constexpr int W = LW + kAccExtra;
    const int N = 1 << d.logN;
    const int logN1 = int(d.logN) - int(d.logN2);
    const int N2 = N >> logN1;
    const int T = N < kTile ? N : kTile;
    const int C = T >> logN1;
    const int k = int(d.k), L = int(d.L);
    const int j0 = tile * C;

    uint64_t* s_res = reinterpret_cast<uint64_t*>(smem);
    uint8_t* cur = smem + smax(size_t(kTile) * 8 * size_t(k), size_t(kTile) * kMaxL * 4);
    uint32_t* s_mq = reinterpret_cast<uint32_t*>(cur);
    cur += size_t(k) * kMqStride * 4;
    uint64_t* s_y = reinterpret_cast<uint64_t*>(cur);
    uint64_t* s_ys = s_y + k;
    uint64_t* s_p = s_ys + k;
    cur += size_t(k) * 8 * 3;
    uint32_t* s_negm = reinterpret_cast<uint32_t*>(cur);
    uint32_t* s_q = s_negm + kMqStride;
    uint32_t* s_mu = s_q + kMqStride;

    __syncthreads();  // shared memory of a previous item is free
    const QConst* qc = d.qc;
    for (int w = threadIdx.x; w < k * kMqStride; w += blockDim.x) s_mq[w] = __ldg(qc->mq + w);
    for (int w = threadIdx.x; w < k; w += blockDim.x) {
        s_y[w] = __ldg(qc->y + w);
        s_ys[w] = __ldg(qc->ys + w);
        s_p[w] = __ldg(t.primes + w);
    }
    for (int w = threadIdx.x; w < kMqStride; w += blockDim.x) {
        s_negm[w] = __ldg(qc->neg_m + w);
        s_q[w] = __ldg(qc->q + w);
    }
    if (threadIdx.x < 4) s_mu[threadIdx.x] = __ldg(qc->mu + threadIdx.x);
    __syncthreads();  // s_p is read by the column stages
    pdl_wait();       // the residues come from the stream's previous kernel

    switch (logN1) {
        case 0: crt_columns<0>(d, t, tile, s_p, s_res); break;
        case 1: crt_columns<1>(d, t, tile, s_p, s_res); break;
        case 2: crt_columns<2>(d, t, tile, s_p, s_res); break;
        case 3: crt_columns<3>(d, t, tile, s_p, s_res); break;
        case 4: crt_columns<4>(d, t, tile, s_p, s_res); break;
        default: crt_columns<5>(d, t, tile, s_p, s_res); break;
    }
    __syncthreads();

    const int tc = threadIdx.x;
    uint32_t r[LW + 1];
    if (tc < T) {
        // acc = acc_lo + acc_hi: the lo and hi halves of the limb products run as two independent
        // carry chains
        uint32_t acc_lo[W], acc_hi[W];
#pragma unroll
        for (int w = 0; w < W; ++w) acc_lo[w] = acc_hi[w] = 0;
        uint64_t frac = 0;
#pragma unroll 1
        for (int i = 0; i < k; ++i) {
            const uint64_t p = c_pc[i].p;
            const uint64_t res = s_res[size_t(i) * T + tc];
            const uint64_t v = csub(shoup_lazy(res, s_y[i], s_ys[i], p), p);  // [0, p)
            frac += (uint64_t(uint32_t(v >> 30)) * c_pc[i].g) >> 31;            // 2^32 v / p_i
            const uint32_t* M = s_mq + i * kMqStride;
            const uint32_t v0 = uint32_t(v), v1 = uint32_t(v >> 32);
            mac_lo<LW, 0, W>(acc_lo, M, v0);
            mac_hi<LW, 1, W>(acc_hi, M, v0);
            mac_lo<LW, 1, W>(acc_lo, M, v1);
            mac_hi<LW, 2, W>(acc_hi, M, v1);
        }
        // acc_lo += round(sum v_i / p_i) * ((-M) mod q)
        const uint32_t kq = uint32_t((frac + (1ull << 31)) >> 32);
        mac_lo<LW, 0, W>(acc_lo, s_negm, kq);
        mac_hi<LW, 1, W>(acc_hi, s_negm, kq);
        asm volatile("add.cc.u32 %0, %0, %1;" : "+r"(acc_lo[0]) : "r"(acc_hi[0]));
#pragma unroll
        for (int w = 1; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, %1;" : "+r"(acc_lo[w]) : "r"(acc_hi[w]));
        asm volatile("addc.u32 %0, %0, %1;" : "+r"(acc_lo[W - 1]) : "r"(acc_hi[W - 1]));
        barrett<LW, W>(acc_lo, s_q, s_mu, int(qc->qbits), r);
    }
    __syncthreads();  // every thread has read s_res; reuse it as output staging
    uint32_t* s_out = reinterpret_cast<uint32_t*>(s_res);
    if (tc < T) {
        uint32_t* o = s_out + tc * L;
        if ((L & 3) == 0) {
#pragma unroll
            for (int l = 0; l < LW; l += 4)
                if (l < L) *reinterpret_cast<uint4*>(o + l) = make_uint4(r[l], r[l + 1], r[l + 2], r[l + 3]);
        } else if ((L & 1) == 0) {
#pragma unroll
            for (int l = 0; l < LW; l += 2)
                if (l < L) *reinterpret_cast<uint2*>(o + l) = make_uint2(r[l], r[l + 1]);
        } else {
#pragma unroll
            for (int l = 0; l < LW; ++l)
                if (l < L) o[l] = r[l];
        }
    }
    __syncthreads();
    store_tile(d.c, N2, L, j0, C, 1 << logN1, s_out);
}

}  // namespace nc
