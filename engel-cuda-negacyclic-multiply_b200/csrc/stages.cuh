// The three stages of one negacyclic product, written as CTA-level device functions so the
// plain per-call kernels and the persistent batched kernel share them.
//
//   stage 1  dec_tile   limbs -> residues mod each prime (solve.cu:533-570 computes the same
//                       residues) and the first log2(N1) forward NTT stages over columns
//   stage 2  row_blocks per (prime, row block of N2 residues): forward NTT of a and of b,
//                       pointwise product, inverse NTT (solve.cu:952-1044, 620-628)
//   stage 3  crt_tile   last log2(N1) inverse stages over columns, then CRT and Barrett
//                       reduction mod q into L limbs (solve.cu:630-642, 752-836)
//
// The NTT is the merged negacyclic form: forward Cooley-Tukey with twiddles psi^bitrev(j)
// (natural order in, bit-reversed order out) and inverse Gentleman-Sande with psi^-bitrev(j)
// (bit-reversed in, natural out), so no twist, untwist or bit-reversal pass exists. N^-1 is
// folded into the CRT constant y_i. Residue rows are k x N u64, prime-major.
#pragma once

#include <cstdint>

#include "arith.cuh"
#include "common.h"

namespace nc {

// Device-wide tables (built once per device). Twiddle entry j of prime i sits at
// fwd[i * kMaxN + j] = (psi^bitrev17(j) ... restricted to the first N), with its Shoup companion.
struct Tables {
    const ulonglong2* fwd;    // [kMaxPrimes][kMaxN]
    const ulonglong2* inv;    // [kMaxPrimes][kMaxN]
    const uint64_t* pow32;    // [kMaxPrimes][kMaxL]  2^(32 l) mod p_i
    const PrimeConst* pc;     // [kMaxPrimes]
};

// ------------------------------------------------------------------------------------------
// shared-memory sizes

__host__ __device__ constexpr size_t dec_smem_bytes() {
    return size_t(kTile) * kMaxL * 4 + size_t(kMaxPrimes) * kMaxL * 8;
}
__host__ __device__ constexpr size_t row_smem_bytes() { return size_t(2) << kRowLogMax << 3; }
__host__ __device__ constexpr size_t crt_smem_bytes(int k) {
    return size_t(kTile) * 8 * (k > 16 ? k : 16)        // residues (>= output staging 256*32*4)
           + size_t(k) * kMqStride * 4                 // M/p_i mod q
           + size_t(k) * 8 * 3                         // y, y shoup, p
           + size_t(k) * 4                             // g
           + size_t(kMqStride) * 4 * 2 + 16;           // -M mod q, q, mu
}
__host__ __device__ constexpr size_t max_smem_bytes() {
    return crt_smem_bytes(kMaxPrimes) > row_smem_bytes()
               ? (crt_smem_bytes(kMaxPrimes) > dec_smem_bytes() ? crt_smem_bytes(kMaxPrimes) : dec_smem_bytes())
               : (row_smem_bytes() > dec_smem_bytes() ? row_smem_bytes() : dec_smem_bytes());
}

// ------------------------------------------------------------------------------------------
// stage 1: residues + forward column stages

template <int LOG_N1>
__device__ __forceinline__ void dec_column(const Tables& t, int i, uint64_t p, uint64_t (&v)[1 << LOG_N1]) {
    constexpr int N1 = 1 << LOG_N1;
    const ulonglong2* tw = t.fwd + size_t(i) * kMaxN;
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

// Sum_l limb_l * 2^(32 l) mod p for one coefficient held in shared memory; result in [0, 2p).
template <int VEC>
__device__ __forceinline__ uint64_t residue_of(const uint32_t* limbs, const uint64_t* pw, int L, uint64_t m) {
    uint32_t a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
    if (VEC == 4) {
#pragma unroll 1
        for (int l = 0; l < L; l += 4) {
            const uint4 x = *reinterpret_cast<const uint4*>(limbs + l);
            const uint64_t c0 = pw[l], c1 = pw[l + 1], c2 = pw[l + 2], c3 = pw[l + 3];
            mac_u32x64(x.x, uint32_t(c0), uint32_t(c0 >> 32), a0, a1, a2, b0, b1, b2);
            mac_u32x64(x.y, uint32_t(c1), uint32_t(c1 >> 32), a0, a1, a2, b0, b1, b2);
            mac_u32x64(x.z, uint32_t(c2), uint32_t(c2 >> 32), a0, a1, a2, b0, b1, b2);
            mac_u32x64(x.w, uint32_t(c3), uint32_t(c3 >> 32), a0, a1, a2, b0, b1, b2);
        }
    } else if (VEC == 2) {
#pragma unroll 1
        for (int l = 0; l < L; l += 2) {
            const uint2 x = *reinterpret_cast<const uint2*>(limbs + l);
            const uint64_t c0 = pw[l], c1 = pw[l + 1];
            mac_u32x64(x.x, uint32_t(c0), uint32_t(c0 >> 32), a0, a1, a2, b0, b1, b2);
            mac_u32x64(x.y, uint32_t(c1), uint32_t(c1 >> 32), a0, a1, a2, b0, b1, b2);
        }
    } else {
#pragma unroll 1
        for (int l = 0; l < L; ++l) {
            const uint64_t c0 = pw[l];
            mac_u32x64(limbs[l], uint32_t(c0), uint32_t(c0 >> 32), a0, a1, a2, b0, b1, b2);
        }
    }
    // S = (a2:a1:a0) + (b2:b1:b0) * 2^32 < 2^99
    const uint64_t lo_a = (uint64_t(a1) << 32) | a0;
    const uint64_t mid = uint64_t(b1) << 32 | b0;  // contributes mid * 2^32
    const uint64_t add_lo = mid << 32;
    const uint64_t lo = lo_a + add_lo;
    const uint64_t hi = uint64_t(a2) + (mid >> 32) + (uint64_t(b2) << 32) + (lo < lo_a ? 1u : 0u);
    return reduce_special(hi, lo, m);
}

template <int LOG_N1>
__device__ void dec_tile(const ProductDesc& d, const Tables& t, int operand, int tile, uint8_t* smem) {
    constexpr int N1 = 1 << LOG_N1;
    const int N = 1 << d.logN;
    const int N2 = N >> LOG_N1;
    const int T = N < kTile ? N : kTile;
    const int C = T >> LOG_N1;
    const int L = int(d.L), k = int(d.k);
    const uint32_t* x = operand ? d.b : d.a;
    uint64_t* R = operand ? d.rb : d.ra;
    uint32_t* s_in = reinterpret_cast<uint32_t*>(smem);
    uint64_t* s_pow = reinterpret_cast<uint64_t*>(smem + size_t(kTile) * kMaxL * 4);
    const int j0 = tile * C;
    const int seg = C * L;

    __syncthreads();  // the previous user of shared memory (persistent CTAs) is done
    for (int u = 0; u < N1; ++u) {
        const size_t first = (size_t(u) * N2 + j0) * L;
        const uint32_t* src = x + first;
        uint32_t* dst = s_in + u * seg;
        if (((first | size_t(seg)) & 3) == 0) {
            const uint4* s4 = reinterpret_cast<const uint4*>(src);
            uint4* d4 = reinterpret_cast<uint4*>(dst);
            for (int w = threadIdx.x; w < (seg >> 2); w += kThreads) d4[w] = __ldg(s4 + w);
        } else {
            for (int w = threadIdx.x; w < seg; w += kThreads) dst[w] = __ldg(src + w);
        }
    }
    for (int w = threadIdx.x; w < k * L; w += kThreads) {
        const int i = w / L, l = w - i * L;
        s_pow[w] = __ldg(t.pow32 + i * kMaxL + l);
    }
    __syncthreads();

    for (int w = threadIdx.x; w < k * C; w += kThreads) {
        const int i = w / C, j = w - i * C;
        const uint64_t p = __ldg(&t.pc[i].p), m = __ldg(&t.pc[i].m);
        const uint64_t* pw = s_pow + i * L;
        uint64_t v[N1];
#pragma unroll
        for (int u = 0; u < N1; ++u) {
            const uint32_t* limbs = s_in + u * seg + j * L;
            if ((L & 3) == 0)
                v[u] = residue_of<4>(limbs, pw, L, m);
            else if ((L & 1) == 0)
                v[u] = residue_of<2>(limbs, pw, L, m);
            else
                v[u] = residue_of<1>(limbs, pw, L, m);
        }
        dec_column<LOG_N1>(t, i, p, v);
        uint64_t* row = R + size_t(i) * N + j0 + j;
#pragma unroll
        for (int u = 0; u < N1; ++u) row[size_t(u) * N2] = v[u];
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

template <int LOG_N2>
struct RowShape {
    static constexpr int N2 = 1 << LOG_N2;
    static constexpr int LOG_E = LOG_N2 < 4 ? LOG_N2 : 4;
    static constexpr int E = 1 << LOG_E;
    static constexpr int T = N2 / E;                     // threads per row block
    static constexpr int ROWS = kThreads / T;            // row blocks per CTA
    static constexpr int NPASS = (LOG_N2 + LOG_E - 1) / LOG_E;
    __host__ __device__ static constexpr int l0(int pass) { return pass * LOG_E; }
    __host__ __device__ static constexpr int r(int pass) {
        return (LOG_N2 - pass * LOG_E) < LOG_E ? (LOG_N2 - pass * LOG_E) : LOG_E;
    }
    __host__ __device__ static constexpr int lolog(int pass) { return LOG_N2 - l0(pass) - r(pass); }
};

// Element index (inside the row block) of register slot e in pass `pass` for thread lt.
template <int LOG_N2, int PASS>
__device__ __forceinline__ int row_index(int lt, int e) {
    using S = RowShape<LOG_N2>;
    constexpr int R = S::r(PASS), LL = S::lolog(PASS);
    const int q = e >> R, s = e & ((1 << R) - 1);
    const int g = lt + S::T * q;
    const int hi = g >> LL, lo = g & ((1 << LL) - 1);
    return (hi << (LOG_N2 - S::l0(PASS))) + (s << LL) + lo;
}

template <int LOG_N2, int PASS, bool FWD>
__device__ __forceinline__ void row_pass(uint64_t (&v)[RowShape<LOG_N2>::E], const ulonglong2* tw, int base, int lt,
                                         uint64_t p) {
    using S = RowShape<LOG_N2>;
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
            const int twbase = (base << (L0 + j)) + (hi << j);
#pragma unroll
            for (int blk = 0; blk < (1 << j); ++blk) {
                const ulonglong2 w = __ldg(tw + twbase + blk);
#pragma unroll
                for (int s0 = 0; s0 < half; ++s0) {
                    const int s = blk * 2 * half + s0;
                    const int e = q * (1 << R) + s;
                    if (FWD)
                        ct_bfly(v[e], v[e + half], w.x, w.y, p, p2);
                    else
                        gs_bfly(v[e], v[e + half], w.x, w.y, p, p2);
                }
            }
        }
    }
}

template <int LOG_N2, int PASS>
__device__ __forceinline__ void row_store(const uint64_t (&v)[RowShape<LOG_N2>::E], uint64_t* buf, int lt) {
    using S = RowShape<LOG_N2>;
    if (S::lolog(PASS) == 0 && S::r(PASS) >= 1) {
#pragma unroll
        for (int e = 0; e < S::E; e += 2) {
            const int x = row_index<LOG_N2, PASS>(lt, e);
            reinterpret_cast<ulonglong2*>(buf)[swz(x) >> 1] = make_ulonglong2(v[e], v[e + 1]);
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) buf[swz(row_index<LOG_N2, PASS>(lt, e))] = v[e];
    }
}

template <int LOG_N2, int PASS>
__device__ __forceinline__ void row_load(uint64_t (&v)[RowShape<LOG_N2>::E], const uint64_t* buf, int lt) {
    using S = RowShape<LOG_N2>;
    if (S::lolog(PASS) == 0 && S::r(PASS) >= 1) {
#pragma unroll
        for (int e = 0; e < S::E; e += 2) {
            const int x = row_index<LOG_N2, PASS>(lt, e);
            const ulonglong2 pr = reinterpret_cast<const ulonglong2*>(buf)[swz(x) >> 1];
            v[e] = pr.x;
            v[e + 1] = pr.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = buf[swz(row_index<LOG_N2, PASS>(lt, e))];
    }
}

// Forward passes 0..NPASS-1 starting from registers in pass-0 layout; ends in last-pass layout.
template <int LOG_N2, int PASS>
__device__ __forceinline__ void row_forward_from(uint64_t (&v)[RowShape<LOG_N2>::E], uint64_t* buf,
                                                 const ulonglong2* tw, int base, int lt, uint64_t p) {
    using S = RowShape<LOG_N2>;
    row_pass<LOG_N2, PASS, true>(v, tw, base, lt, p);
    if constexpr (PASS + 1 < S::NPASS) {
        __syncthreads();
        row_store<LOG_N2, PASS>(v, buf, lt);
        __syncthreads();
        row_load<LOG_N2, PASS + 1>(v, buf, lt);
        row_forward_from<LOG_N2, PASS + 1>(v, buf, tw, base, lt, p);
    }
}

// Inverse passes PASS..0 starting from registers in pass-PASS layout; ends in pass-0 layout.
template <int LOG_N2, int PASS>
__device__ __forceinline__ void row_inverse_from(uint64_t (&v)[RowShape<LOG_N2>::E], uint64_t* buf,
                                                 const ulonglong2* tw, int base, int lt, uint64_t p) {
    row_pass<LOG_N2, PASS, false>(v, tw, base, lt, p);
    if constexpr (PASS > 0) {
        __syncthreads();
        row_store<LOG_N2, PASS>(v, buf, lt);
        __syncthreads();
        row_load<LOG_N2, PASS - 1>(v, buf, lt);
        row_inverse_from<LOG_N2, PASS - 1>(v, buf, tw, base, lt, p);
    }
}

// One CTA handles ROWS row blocks: block rb = item * ROWS + (tid / T) is prime rb >> logN1,
// row u = rb & (N1 - 1), residues [u * N2, (u + 1) * N2) of that prime's row.
template <int LOG_N2>
__device__ void row_blocks(const ProductDesc& d, const Tables& t, int item, uint8_t* smem) {
    using S = RowShape<LOG_N2>;
    constexpr int LAST = S::NPASS - 1;
    const int logN1 = int(d.logN) - LOG_N2;
    const int N = 1 << d.logN;
    const int rr = threadIdx.x / S::T, lt = threadIdx.x - rr * S::T;
    const int rb = item * S::ROWS + rr;
    const bool active = rb < (int(d.k) << logN1);
    const int i = active ? rb >> logN1 : 0;
    const int u = rb & ((1 << logN1) - 1);
    const uint64_t p = __ldg(&t.pc[i].p), m = __ldg(&t.pc[i].m);
    const int base = (1 << logN1) + u;  // (N1 + u): twiddle index of local stage l is base << l + ...
    const size_t off = size_t(i) * N + size_t(u) * S::N2;
    uint64_t* buf = reinterpret_cast<uint64_t*>(smem) + rr * S::N2;
    uint64_t* buf_a = reinterpret_cast<uint64_t*>(smem) + (size_t(S::ROWS) << LOG_N2) + rr * S::N2;
    const ulonglong2* twf = t.fwd + size_t(i) * kMaxN;
    const ulonglong2* twi = t.inv + size_t(i) * kMaxN;
    uint64_t v[S::E];

    __syncthreads();  // shared memory of a previous item is free
    if (d.mode == kModeCachedA) {
        // a is already in the NTT domain: stage it into buf_a
#pragma unroll
        for (int e = 0; e < S::E; ++e) {
            const int x = row_index<LOG_N2, 0>(lt, e);
            buf_a[swz(x)] = active ? __ldcg(d.a_hat + off + x) : 0;
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = active ? __ldcg(d.ra + off + row_index<LOG_N2, 0>(lt, e)) : 0;
        row_forward_from<LOG_N2, 0>(v, buf, twf, base, lt, p);
        if (d.mode == kModeForward) {
            __syncthreads();
            row_store<LOG_N2, LAST>(v, buf, lt);
            __syncthreads();
            row_load<LOG_N2, 0>(v, buf, lt);
            if (active) {
#pragma unroll
                for (int e = 0; e < S::E; ++e) __stcg(d.hat_out + off + row_index<LOG_N2, 0>(lt, e), v[e]);
            }
            return;
        }
        row_store<LOG_N2, LAST>(v, buf_a, lt);
    }
#pragma unroll
    for (int e = 0; e < S::E; ++e) v[e] = active ? __ldcg(d.rb + off + row_index<LOG_N2, 0>(lt, e)) : 0;
    row_forward_from<LOG_N2, 0>(v, buf, twf, base, lt, p);
    __syncthreads();
    {
        uint64_t av[S::E];
        row_load<LOG_N2, LAST>(av, buf_a, lt);
        const uint64_t p2 = 2 * p;
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = mulmod_special(csub(csub(av[e], p2), p), v[e], m);
    }
    row_inverse_from<LOG_N2, LAST>(v, buf, twi, base, lt, p);
    if (active) {
#pragma unroll
        for (int e = 0; e < S::E; ++e) __stcg(d.ra + off + row_index<LOG_N2, 0>(lt, e), v[e]);
    }
}

// ------------------------------------------------------------------------------------------
// stage 3: inverse column stages + CRT + Barrett

template <int LOG_N1>
__device__ void crt_columns(const ProductDesc& d, const Tables& t, int tile, uint64_t* s_res) {
    constexpr int N1 = 1 << LOG_N1;
    const int N = 1 << d.logN;
    const int N2 = N >> LOG_N1;
    const int T = N < kTile ? N : kTile;
    const int C = T >> LOG_N1;
    const int k = int(d.k);
    const int j0 = tile * C;
    for (int w = threadIdx.x; w < k * C; w += kThreads) {
        const int i = w / C, j = w - i * C;
        const uint64_t p = __ldg(&t.pc[i].p);
        const uint64_t p2 = 2 * p;
        const uint64_t* row = d.ra + size_t(i) * N + j0 + j;
        uint64_t v[N1];
#pragma unroll
        for (int u = 0; u < N1; ++u) v[u] = __ldcg(row + size_t(u) * N2);
        const ulonglong2* tw = t.inv + size_t(i) * kMaxN;
#pragma unroll
        for (int s = LOG_N1 - 1; s >= 0; --s) {
            const int half = N1 >> (s + 1);
#pragma unroll
            for (int blk = 0; blk < (1 << s); ++blk) {
                const ulonglong2 wv = __ldg(tw + (1 << s) + blk);
#pragma unroll
                for (int jj = 0; jj < half; ++jj) {
                    const int uu = blk * 2 * half + jj;
                    gs_bfly(v[uu], v[uu + half], wv.x, wv.y, p, p2);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < N1; ++u) s_res[size_t(i) * T + u * C + j] = v[u];
    }
}

// acc[OFF..W) += v * M[0..LW)  (carry chains; the top word absorbs the final carry)
template <int LW, int OFF, int W>
__device__ __forceinline__ void mac_row(uint32_t (&acc)[W], const uint32_t* M, uint32_t v) {
    asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF]) : "r"(v), "r"(M[0]));
#pragma unroll
    for (int l = 1; l < LW; ++l) asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF + l]) : "r"(v), "r"(M[l]));
#pragma unroll
    for (int w = OFF + LW; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, 0;" : "+r"(acc[w]));
    asm volatile("addc.u32 %0, %0, 0;" : "+r"(acc[W - 1]));
    asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF + 1]) : "r"(v), "r"(M[0]));
#pragma unroll
    for (int l = 1; l < LW; ++l)
        asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(acc[OFF + 1 + l]) : "r"(v), "r"(M[l]));
#pragma unroll
    for (int w = OFF + 1 + LW; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, 0;" : "+r"(acc[w]));
    if (OFF + 1 + LW < W) asm volatile("addc.u32 %0, %0, 0;" : "+r"(acc[W - 1]));
}

__device__ __forceinline__ uint32_t funnel(uint32_t lo, uint32_t hi, int sh) {
    return __funnelshift_r(lo, hi, sh);
}

// r (LW + 1 words) := acc mod q, for acc < 2^(qbits + kBarrettT). q_top = index of q's top word.
template <int LW, int W>
__device__ __forceinline__ void barrett(uint32_t (&acc)[W], const uint32_t* q, const uint32_t* mu, int qbits,
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
    const uint32_t m0 = mu[0], m1 = mu[1], m2 = mu[2];
    uint32_t t[6] = {0, 0, 0, 0, 0, 0};
    {
        const uint32_t ys[3] = {y0, y1, y2};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            uint64_t carry = 0;
            const uint32_t ms[3] = {m0, m1, m2};
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) {
                const uint64_t cur = uint64_t(t[a + bb]) + uint64_t(ys[a]) * ms[bb] + carry;
                t[a + bb] = uint32_t(cur);
                carry = cur >> 32;
            }
            t[a + 3] = uint32_t(carry);
        }
    }
    const uint32_t q0 = funnel(t[2], t[3], 7), q1 = funnel(t[3], t[4], 7), q2 = funnel(t[4], t[5], 7);
    // prod = (q2:q1:q0) * q, low LW + 1 words
    uint32_t prod[LW + 1];
#pragma unroll
    for (int w = 0; w <= LW; ++w) prod[w] = 0;
    {
        const uint32_t qs[3] = {q0, q1, q2};
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
    const int logN1 = int(d.logN) > kRowLogMax ? int(d.logN) - kRowLogMax : 0;
    const int N2 = N >> logN1;
    const int T = N < kTile ? N : kTile;
    const int C = T >> logN1;
    const int k = int(d.k), L = int(d.L);
    const int j0 = tile * C;

    uint64_t* s_res = reinterpret_cast<uint64_t*>(smem);
    uint8_t* cur = smem + size_t(kTile) * 8 * (k > 16 ? k : 16);
    uint32_t* s_mq = reinterpret_cast<uint32_t*>(cur);
    cur += size_t(k) * kMqStride * 4;
    uint64_t* s_y = reinterpret_cast<uint64_t*>(cur);
    uint64_t* s_ys = s_y + k;
    uint64_t* s_p = s_ys + k;
    cur += size_t(k) * 8 * 3;
    uint32_t* s_g = reinterpret_cast<uint32_t*>(cur);
    cur += size_t(k) * 4;
    uint32_t* s_negm = reinterpret_cast<uint32_t*>(cur);
    uint32_t* s_q = s_negm + kMqStride;
    uint32_t* s_mu = s_q + kMqStride;

    __syncthreads();  // shared memory of a previous item is free
    const QConst* qc = d.qc;
    for (int w = threadIdx.x; w < k * kMqStride; w += kThreads) s_mq[w] = __ldg(qc->mq + w);
    for (int w = threadIdx.x; w < k; w += kThreads) {
        s_y[w] = __ldg(qc->y + w);
        s_ys[w] = __ldg(qc->ys + w);
        s_p[w] = __ldg(&t.pc[w].p);
        s_g[w] = __ldg(&t.pc[w].g);
    }
    for (int w = threadIdx.x; w < kMqStride; w += kThreads) {
        s_negm[w] = __ldg(qc->neg_m + w);
        s_q[w] = __ldg(qc->q + w);
    }
    if (threadIdx.x < 4) s_mu[threadIdx.x] = __ldg(qc->mu + threadIdx.x);

    switch (logN1) {
        case 0: crt_columns<0>(d, t, tile, s_res); break;
        case 1: crt_columns<1>(d, t, tile, s_res); break;
        case 2: crt_columns<2>(d, t, tile, s_res); break;
        case 3: crt_columns<3>(d, t, tile, s_res); break;
        default: crt_columns<4>(d, t, tile, s_res); break;
    }
    __syncthreads();

    const int tc = threadIdx.x;
    uint32_t r[LW + 1];
    if (tc < T) {
        uint32_t acc[W];
#pragma unroll
        for (int w = 0; w < W; ++w) acc[w] = 0;
        uint64_t frac = 0;
#pragma unroll 1
        for (int i = 0; i < k; ++i) {
            const uint64_t p = s_p[i];
            const uint64_t res = s_res[size_t(i) * T + tc];
            const uint64_t v = csub(shoup_lazy(res, s_y[i], s_ys[i], p), p);  // [0, p)
            frac += (uint64_t(uint32_t(v >> 30)) * s_g[i]) >> 31;              // 2^32 v / p_i
            const uint32_t* M = s_mq + i * kMqStride;
            mac_row<LW, 0, W>(acc, M, uint32_t(v));
            mac_row<LW, 1, W>(acc, M, uint32_t(v >> 32));
        }
        // acc += round(sum v_i / p_i) * ((-M) mod q)
        const uint32_t kq = uint32_t((frac + (1ull << 31)) >> 32);
        {
            uint32_t lo_part[LW];
#pragma unroll
            for (int l = 0; l < LW; ++l) lo_part[l] = s_negm[l];
            mac_row<LW, 0, W>(acc, lo_part, kq);
        }
        barrett<LW, W>(acc, s_q, s_mu, int(d.qc->qbits), r);
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
    const int N1 = 1 << logN1;
    const int seg = C * L;
    for (int u = 0; u < N1; ++u) {
        const size_t first = (size_t(u) * N2 + j0) * L;
        uint32_t* dst = d.c + first;
        const uint32_t* src = s_out + u * seg;
        if (((first | size_t(seg)) & 3) == 0) {
            uint4* d4 = reinterpret_cast<uint4*>(dst);
            const uint4* s4 = reinterpret_cast<const uint4*>(src);
            for (int w = threadIdx.x; w < (seg >> 2); w += kThreads) d4[w] = s4[w];
        } else {
            for (int w = threadIdx.x; w < seg; w += kThreads) dst[w] = src[w];
        }
    }
}

}  // namespace nc
