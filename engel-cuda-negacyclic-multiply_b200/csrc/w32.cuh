// The 30-bit word engine: residues modulo primes p < 2^30 with p = 1 (mod 2^17), one 32-bit word
// each, for the plain product of two operands.
//
// A 62-bit residue costs a 64 x 64-bit Shoup product per butterfly (about 17 integer multiply-adds
// and as many ALU operations on the GPU's 32-bit datapath); a 30-bit residue costs one
// multiply-high and two multiply-lows. Twice as many primes cover the same bound, so a product
// does twice the butterflies at about a third of the instructions each. The stages and their
// order are those of the 62-bit engine (stages.cuh): residues + forward column stages, row
// blocks (forward a, forward b, pointwise, inverse), inverse column stages + CRT. Values stay
// lazily reduced: forward (Cooley-Tukey) butterflies in [0, 4p), inverse (Gentleman-Sande) in
// [0, 2p), which 4p < 2^32 allows. The pointwise product is a Montgomery product (its 2^-32 is
// folded into the CRT constant of each prime).
#pragma once

#include <cstdint>

#include "stages.cuh"

namespace nc {

namespace w32 {

// x - m if x >= m, else x, for x < 2m <= 2^31 (x - m wraps above x when x < m).
__device__ __forceinline__ uint32_t csub(uint32_t x, uint32_t m) { return min(x, x - m); }

// y w mod p in [0, 2p) for any y < 2^32 and w < p, with wq = floor(w 2^32 / p).
__device__ __forceinline__ uint32_t shoup(uint32_t y, uint32_t w, uint32_t wq, uint32_t p) {
    return y * w - __umulhi(y, wq) * p;
}

// Forward butterfly (x, y) -> (x + w y, x - w y); inputs and outputs in [0, 4p).
__device__ __forceinline__ void ct_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p, uint32_t p2) {
    const uint32_t u = csub(x, p2);
    const uint32_t t = shoup(y, w, wq, p);
    x = u + t;
    y = u - t + p2;
}

// Inverse butterfly (x, y) -> (x + y, (x - y) w); inputs and outputs in [0, 2p).
__device__ __forceinline__ void gs_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p, uint32_t p2) {
    const uint32_t s = csub(x + y, p2);
    const uint32_t d = x - y + p2;
    x = s;
    y = shoup(d, w, wq, p);
}

// The inverse butterfly with twiddle -w: (x, y) -> (x + y, (y - x) w). The row stage's inverse
// twiddles are negated forward ones (below), so it takes the forward pair unchanged.
__device__ __forceinline__ void gs_bfly_neg(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p, uint32_t p2) {
    const uint32_t s = csub(x + y, p2);
    const uint32_t d = y - x + p2;
    x = s;
    y = shoup(d, w, wq, p);
}

// a b 2^-32 mod p in [0, 2p) for a < p, b < 4p (Montgomery; pinv = -p^-1 mod 2^32): the sum
// a b + m p stays below 2^63 and its high word below p (4 p^2 / 2^32) + p.
__device__ __forceinline__ uint32_t mont(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    const uint64_t t = uint64_t(a) * b;
    const uint32_t m = uint32_t(t) * pinv;
    return uint32_t((t + uint64_t(m) * p) >> 32);
}

// 16-byte-chunk XOR swizzle inside 128-byte rows of a u32 buffer (four words a chunk).
__device__ __forceinline__ int swz(int x) {
    const int c = x >> 2;
    const int pc = (c & ~7) | ((c ^ (c >> 3)) & 7);
    return (pc << 2) | (x & 3);
}

// ------------------------------------------------------------------------------------------
// column stages (registers), as column_forward / column_inverse of the 62-bit engine

template <int LOG_N1>
__device__ __forceinline__ void column_forward_root(const uint2* tw, int root, uint32_t p, uint32_t (&v)[1 << LOG_N1]) {
    constexpr int N1 = 1 << LOG_N1;
    const uint32_t p2 = 2 * p;
#pragma unroll
    for (int s = 0; s < LOG_N1; ++s) {
        const int half = N1 >> (s + 1);
#pragma unroll
        for (int blk = 0; blk < (1 << s); ++blk) {
            const uint2 w = __ldg(tw + (root << s) + blk);
#pragma unroll
            for (int jj = 0; jj < half; ++jj) {
                const int u = blk * 2 * half + jj;
                ct_bfly(v[u], v[u + half], w.x, w.y, p, p2);
            }
        }
    }
}

template <int LOG_N1>
__device__ __forceinline__ void column_inverse_root(const uint2* tw, int root, uint32_t p, uint32_t (&v)[1 << LOG_N1]) {
    constexpr int N1 = 1 << LOG_N1;
    const uint32_t p2 = 2 * p;
#pragma unroll
    for (int s = LOG_N1 - 1; s >= 0; --s) {
        const int half = N1 >> (s + 1);
#pragma unroll
        for (int blk = 0; blk < (1 << s); ++blk) {
            const uint2 w = __ldg(tw + (root << s) + blk);
#pragma unroll
            for (int jj = 0; jj < half; ++jj) {
                const int u = blk * 2 * half + jj;
                gs_bfly(v[u], v[u + half], w.x, w.y, p, p2);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// row blocks: the register passes of stages.cuh over u32 residues

// One pass of R stages over the thread's groups. tw is a row block's staged twiddles (local
// stage l at tw[(1 << l) + t], stage_twiddles). Forward passes take entry t of the row block's
// forward table; inverse passes take the staged forward twiddles of the mirrored row block in
// reverse order: the inverse twiddle of node 2^s + j of the merged tree, psi^-bitrev(2^s + j),
// equals -psi^bitrev(2^s + (2^s - 1 - j)) (psi^N = -1), and for a row block u of N1 at local
// stage l, j = u 2^l + t mirrors to (N1 - 1 - u) 2^l + (2^l - 1 - t). The 2^j twiddles of a
// stage are adjacent, so pairs of them load as one 16-byte access.
template <class S, int PASS, bool FWD>
__device__ __forceinline__ void row_pass(uint32_t (&v)[S::E], const uint2* tw, int lt, uint32_t p) {
    constexpr int R = S::r(PASS), LL = S::lolog(PASS), L0 = S::l0(PASS);
    const uint32_t p2 = 2 * p;
#pragma unroll
    for (int q = 0; q < (S::E >> R); ++q) {
        const int g = lt + S::T * q;
        const int hi = g >> LL;
#pragma unroll
        for (int jj = 0; jj < R; ++jj) {
            const int j = FWD ? jj : R - 1 - jj;
            const int half = 1 << (R - 1 - j);
            uint2 w[1 << (R - 1)];
            if (FWD) {
                // entries (1 << l) + hi 2^j + blk
                const int first = (1 << (L0 + j)) + (hi << j);
                if (j == 0) {
                    w[0] = tw[first];
                } else {
#pragma unroll
                    for (int b2 = 0; b2 < (1 << j); b2 += 2) {
                        const uint4 pr = reinterpret_cast<const uint4*>(tw)[(first + b2) >> 1];
                        w[b2] = make_uint2(pr.x, pr.y);
                        w[b2 + 1] = make_uint2(pr.z, pr.w);
                    }
                }
            } else {
                // entries (2 << l) - 1 - hi 2^j - blk (descending in blk)
                const int last = (2 << (L0 + j)) - 1 - (hi << j);
                if (j == 0) {
                    w[0] = tw[last];
                } else {
#pragma unroll
                    for (int b2 = 0; b2 < (1 << j); b2 += 2) {
                        const uint4 pr = reinterpret_cast<const uint4*>(tw)[(last - b2 - 1) >> 1];
                        w[b2] = make_uint2(pr.z, pr.w);
                        w[b2 + 1] = make_uint2(pr.x, pr.y);
                    }
                }
            }
#pragma unroll
            for (int blk = 0; blk < (1 << j); ++blk) {
#pragma unroll
                for (int s0 = 0; s0 < half; ++s0) {
                    const int e = q * (1 << R) + blk * 2 * half + s0;
                    if (FWD)
                        ct_bfly(v[e], v[e + half], w[blk].x, w[blk].y, p, p2);
                    else
                        gs_bfly_neg(v[e], v[e + half], w[blk].x, w[blk].y, p, p2);
                }
            }
        }
    }
}

// A thread's values of pass PASS to / from the row buffer. When the pass's groups are runs of
// consecutive elements (lolog 0), each run of four (or two) goes as one 16-byte (8-byte) access.
template <class S, int PASS>
__device__ __forceinline__ void row_store(const uint32_t (&v)[S::E], uint32_t* buf, int lt) {
    if constexpr (S::lolog(PASS) == 0 && S::r(PASS) >= 2) {
#pragma unroll
        for (int e = 0; e < S::E; e += 4) {
            const int x = row_index<S, PASS>(lt, e);
            reinterpret_cast<uint4*>(buf)[swz(x) >> 2] = make_uint4(v[e], v[e + 1], v[e + 2], v[e + 3]);
        }
    } else if constexpr (S::lolog(PASS) == 0 && S::r(PASS) == 1) {
#pragma unroll
        for (int e = 0; e < S::E; e += 2) {
            const int x = row_index<S, PASS>(lt, e);
            reinterpret_cast<uint2*>(buf)[swz(x) >> 1] = make_uint2(v[e], v[e + 1]);
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) buf[swz(row_index<S, PASS>(lt, e))] = v[e];
    }
}

template <class S, int PASS>
__device__ __forceinline__ void row_load(uint32_t (&v)[S::E], const uint32_t* buf, int lt) {
    if constexpr (S::lolog(PASS) == 0 && S::r(PASS) >= 2) {
#pragma unroll
        for (int e = 0; e < S::E; e += 4) {
            const uint4 q = reinterpret_cast<const uint4*>(buf)[swz(row_index<S, PASS>(lt, e)) >> 2];
            v[e] = q.x;
            v[e + 1] = q.y;
            v[e + 2] = q.z;
            v[e + 3] = q.w;
        }
    } else if constexpr (S::lolog(PASS) == 0 && S::r(PASS) == 1) {
#pragma unroll
        for (int e = 0; e < S::E; e += 2) {
            const uint2 q = reinterpret_cast<const uint2*>(buf)[swz(row_index<S, PASS>(lt, e)) >> 1];
            v[e] = q.x;
            v[e + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = buf[swz(row_index<S, PASS>(lt, e))];
    }
}

template <class S, int PASS>
__device__ __forceinline__ void row_forward_from(uint32_t (&v)[S::E], uint32_t* buf, const uint2* tw, int lt, uint32_t p) {
    row_pass<S, PASS, true>(v, tw, lt, p);
    if constexpr (PASS + 1 < S::NPASS) {
        __syncthreads();
        row_store<S, PASS>(v, buf, lt);
        __syncthreads();
        row_load<S, PASS + 1>(v, buf, lt);
        row_forward_from<S, PASS + 1>(v, buf, tw, lt, p);
    }
}

template <class S, int PASS>
__device__ __forceinline__ void row_inverse_from(uint32_t (&v)[S::E], uint32_t* buf, const uint2* tw, int lt, uint32_t p) {
    row_pass<S, PASS, false>(v, tw, lt, p);
    if constexpr (PASS > 0) {
        __syncthreads();
        row_store<S, PASS>(v, buf, lt);
        __syncthreads();
        row_load<S, PASS - 1>(v, buf, lt);
        row_inverse_from<S, PASS - 1>(v, buf, tw, lt, p);
    }
}

// 512-thread row CTAs (two per SM) also prefetch operand b's residue block into shared memory;
// 256-thread ones (four per SM) have no room left for it.
NC_HD constexpr bool row_prefetch_b(int threads) { return threads == 512; }

// Dynamic shared memory of a row CTA: the row buffer, the buffer of operand a's transform and,
// with row_prefetch_b, b's residue block (4 bytes a residue each), then each row block's forward
// and inverse twiddles (8 bytes an entry, N2 entries each).
NC_HD constexpr size_t row_smem_bytes(int threads, int logE) {
    return size_t(threads) * (size_t(1) << logE) * (row_prefetch_b(threads) ? 28 : 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Bounded wait for phase `parity` of the mbarrier at shared address `bar`: false if it did not
// complete within 2^22 polls.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The twiddles of the row block under node `base` of the merged tree: local stage l uses the 2^l
// entries tw[(base << l) + t], stored at s[(1 << l) + t] (entry 0 unused), so that the row passes
// read them from shared memory with base 1. Stages l >= 1 go as bulk copies (2^l entries of 8
// bytes: 16-byte aligned and a multiple of 16 bytes at both ends) that complete on the mbarrier
// `bar`; stage 0's single entry as a plain load.
template <int LOG_N2>
__device__ __forceinline__ void stage_twiddles(const uint2* tw, int base, uint2* s, uint32_t bar) {
    s[1] = __ldg(tw + base);
#pragma unroll
    for (int l = 1; l < LOG_N2; ++l)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(s + (1 << l))),
                     "l"(tw + (size_t(base) << l)), "r"(8u << l), "r"(bar)
                     : "memory");
}

// The same entries by plain loads, every thread of the CTA taking its share (the fallback if the
// bulk copies do not complete in time).
template <int LOG_N2>
__device__ __forceinline__ void copy_twiddles(const uint2* tw, int base, uint2* s, int part, int parts) {
    for (int e = 1 + part; e < (1 << LOG_N2); e += parts) {
        const int l = 31 - __clz(e);
        s[e] = __ldg(tw + (size_t(base) << l) + (e - (1 << l)));
    }
}

// One CTA of THREADS threads handles THREADS / T row blocks, as row_blocks of stages.cuh: block
// rb = item * ROWS + (tid / T) is prime rb >> logN1, row u = rb & (N1 - 1). Modes: product
// (forward a and b, pointwise, inverse), cached-a (a's transform read from a_hat), forward (a's
// transform written to hat_out). Residues are k x N u32. The twiddles and the residue blocks of
// each row block are staged in shared memory at the start by bulk copies that complete on the
// CTA's mbarrier `bar` (row_barrier_init), phase `parity` (a persistent CTA's items alternate
// phases): the passes then wait on no global load. use_bulk false (a persistent CTA after a bulk
// wait gave up) loads them with plain loads instead. Returns false if this item's bulk wait gave
// up (its data then came by plain loads, so the item's result stands).
template <int LOG_N2, int LOG_E, int THREADS>
__device__ __forceinline__ void row_barrier_init(uint32_t bar) {
    using S = RowShape<LOG_N2, LOG_E>;
    constexpr int ROWS = THREADS / S::T;
    if (threadIdx.x == 0) {
        // per item: one arrival per row for its twiddles and, for blocks of four and more, one for
        // its residue blocks
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(LOG_N2 >= 2 ? 2 * ROWS : ROWS)
                     : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

template <int LOG_N2, int LOG_E, int THREADS>
__device__ __forceinline__ bool row_blocks(const ProductDesc& d, const Tables& t, int item, uint8_t* smem,
                                           uint32_t bar, uint32_t parity, bool use_bulk) {
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
    const uint32_t p = __ldg(&t.pc32[i].p), pinv = __ldg(&t.pc32[i].pinv);
    // node of the row block in the merged tree, and of its mirror (N1 - 1 - u), whose forward
    // twiddles serve as the inverse ones (row_pass)
    const int base = (1 << logN1) + u;
    const int base_mirror = (2 << logN1) - 1 - u;
    const size_t off = size_t(i) * N + size_t(u) * S::N2;
    constexpr bool PF_B = row_prefetch_b(THREADS);
    constexpr int NBUF = PF_B ? 3 : 2;
    uint32_t* buf = reinterpret_cast<uint32_t*>(smem) + rr * S::N2;
    uint32_t* buf_a = reinterpret_cast<uint32_t*>(smem) + size_t(ROWS) * S::N2 + rr * S::N2;
    uint32_t* b_in = reinterpret_cast<uint32_t*>(smem) + size_t(2) * ROWS * S::N2 + rr * S::N2;  // with PF_B
    uint2* s_twf = reinterpret_cast<uint2*>(smem + size_t(NBUF) * ROWS * S::N2 * 4) + size_t(rr) * 2 * S::N2;
    uint2* s_twi = s_twf + S::N2;
    const uint2* twf = t.fwd32 + size_t(i) * kMaxN;
    const uint32_t* ra = reinterpret_cast<const uint32_t*>(d.ra);
    const uint32_t* rb_res = reinterpret_cast<const uint32_t*>(d.rb);
    const bool inverse = d.mode != kModeForward;
    uint32_t v[S::E];

    __syncthreads();  // shared memory of a previous item is free
    if (use_bulk && lt == 0) {
        // the twiddle tables do not depend on the previous kernel: their copies start before its end
        const uint32_t bytes = (inverse ? 2u : 1u) * 8u * ((1u << LOG_N2) - 2u);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        stage_twiddles<LOG_N2>(twf, base, s_twf, bar);
        if (inverse) stage_twiddles<LOG_N2>(twf, base_mirror, s_twi, bar);
    }
    // every thread waits for the copies (bounded); if any gave up, each row's threads copy its
    // twiddles themselves and, before the item ends, wait once more for the copies in flight
    bool staged = use_bulk;
    auto twiddles_ready = [&] {
        if (use_bulk) staged = __syncthreads_and(bar_wait(bar, parity) ? 1 : 0) != 0;
        if (!staged) {
            copy_twiddles<LOG_N2>(twf, base, s_twf, lt, S::T);
            if (inverse) copy_twiddles<LOG_N2>(twf, base_mirror, s_twi, lt, S::T);
            __syncthreads();
        }
    };
    auto finish = [&] {
        if (use_bulk && !staged) bar_wait(bar, parity);
        return staged || !use_bulk;
    };

    pdl_wait();  // the residues come from the stream's previous kernel
    // the residue blocks as bulk copies too (16-byte aligned for blocks of 4 and more): product
    // and forward modes put a's block in buf_a and (with PF_B) b's in b_in; cached-a mode a_hat's
    // block in buf and b's in buf_a. They are read in the first pass's layout, before any thread
    // writes those buffers again.
    constexpr bool BULK = LOG_N2 >= 2;
    const uint32_t* a_src = d.mode == kModeCachedA ? reinterpret_cast<const uint32_t*>(d.a_hat) + off : ra + off;
    uint32_t* a_dst = d.mode == kModeCachedA ? buf : buf_a;
    uint32_t* b_dst = d.mode == kModeCachedA ? buf_a : b_in;
    const bool b_bulk = d.mode == kModeCachedA || (PF_B && d.mode == kModeProduct);
    if (BULK && use_bulk && lt == 0) {
        asm volatile("fence.proxy.async.global;" ::: "memory");  // the previous kernel's writes -> bulk reads
        const uint32_t bytes = (b_bulk ? 2u : 1u) * 4u * uint32_t(S::N2);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(a_dst)),
                     "l"(a_src), "r"(4u * S::N2), "r"(bar)
                     : "memory");
        if (b_bulk)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             smem_addr(b_dst)),
                         "l"(rb_res + off), "r"(4u * S::N2), "r"(bar)
                         : "memory");
    }
    if (!BULK) {
        // blocks of fewer than four residues: plain loads into the same places
#pragma unroll
        for (int e = 0; e < S::E; ++e) {
            const int x = row_index<S, 0>(lt, e);
            a_dst[x] = __ldcg(a_src + x);
            if (b_bulk) b_dst[x] = __ldcg(rb_res + off + x);
        }
    }
    twiddles_ready();
    if (BULK && !staged) {
        // no bulk copies, or they gave up: each row's threads load its blocks themselves
        for (int x = lt; x < S::N2; x += S::T) {
            a_dst[x] = __ldcg(a_src + x);
            if (b_bulk) b_dst[x] = __ldcg(rb_res + off + x);
        }
        __syncthreads();
    }
    if (d.mode == kModeCachedA) {
        // b's residues to registers, then a_hat from its raw block into buf_a in the last pass's
        // swizzled layout (b's raw block, also in buf_a, is read first)
        uint32_t av[S::E];
#pragma unroll
        for (int e = 0; e < S::E; ++e) {
            const int x = row_index<S, 0>(lt, e);
            v[e] = buf_a[x];
            av[e] = buf[x];
        }
        __syncthreads();
#pragma unroll
        for (int e = 0; e < S::E; ++e) buf_a[swz(row_index<S, 0>(lt, e))] = av[e];
    } else {
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = buf_a[row_index<S, 0>(lt, e)];
        if constexpr (S::NPASS == 1) __syncthreads();  // buf_a's raw block is read before it is rewritten
        row_forward_from<S, 0>(v, buf, s_twf, lt, p);
        if (d.mode == kModeForward) {
            __syncthreads();
            row_store<S, LAST>(v, buf, lt);
            __syncthreads();
            row_load<S, 0>(v, buf, lt);
            if (active) {
                uint32_t* out = reinterpret_cast<uint32_t*>(d.hat_out);
#pragma unroll
                for (int e = 0; e < S::E; ++e) __stcg(out + off + row_index<S, 0>(lt, e), v[e]);
            }
            return finish();
        }
        row_store<S, LAST>(v, buf_a, lt);
        if constexpr (PF_B) {
#pragma unroll
            for (int e = 0; e < S::E; ++e) v[e] = b_in[row_index<S, 0>(lt, e)];
        } else {
#pragma unroll
            for (int e = 0; e < S::E; ++e) v[e] = __ldcg(rb_res + off + row_index<S, 0>(lt, e));
        }
    }
    row_forward_from<S, 0>(v, buf, s_twf, lt, p);
    __syncthreads();
    const uint32_t p2 = 2 * p;
    uint32_t av[S::E];
    row_load<S, LAST>(av, buf_a, lt);
#pragma unroll
    for (int e = 0; e < S::E; ++e) v[e] = mont(csub(csub(av[e], p2), p), v[e], p, pinv);
    row_inverse_from<S, LAST>(v, buf, s_twi, lt, p);
    if (active) {
        uint32_t* out = reinterpret_cast<uint32_t*>(d.ra);
#pragma unroll
        for (int e = 0; e < S::E; ++e) __stcg(out + off + row_index<S, 0>(lt, e), v[e]);
    }
    return finish();
}

// Row pairs of a batch's persistent row launch (plain products, one row block a row of the CTA):
// row block u of a prime and its mirror u' = N1 - 1 - u in turn. The forward twiddles of u' read
// in reverse are the inverse twiddles of u and the other way round (row_pass), so the pair's
// twiddles are staged once, and u''s residue block of a arrives by a bulk copy issued once u's
// pointwise product has read buf_a, while u's inverse runs: one staging wait for two blocks.
// Mbarrier phases (two arrivals each, row_barrier_init): `parity` for the twiddles and u's block
// of a, parity ^ 1 for the block of a of u'; b's blocks come by plain loads in the forward pass,
// as in row_blocks without row_prefetch_b (256-thread CTAs). rb0 and rb1 are the two row blocks
// (prime * N1 + u). Returns false if a bulk wait gave up (the blocks then came by
// plain loads and the results stand); the caller then stops using the barrier. With use_bulk
// false every block comes by plain loads. If the first member's copies have not landed after two
// bounded waits, its buffers cannot safely take the second member's blocks: error[0] is set
// (error[1] = what), which the host reports as a failed batch.
template <int LOG_N2, int LOG_E, int THREADS>
__device__ __forceinline__ bool row_pair(const ProductDesc& d, const Tables& t, int rb0, int rb1, uint8_t* smem,
                                         uint32_t bar, uint32_t parity, bool use_bulk, uint32_t* error, uint32_t what) {
    using S = RowShape<LOG_N2, LOG_E>;
    static_assert(S::T == THREADS && LOG_N2 >= 2, "row pairs take one row block a CTA, staged by bulk copies");
    static_assert(!row_prefetch_b(THREADS), "row pairs load b's blocks in the forward pass");
    constexpr int LAST = S::NPASS - 1;
    const int logN1 = int(d.logN) - LOG_N2;
    const int N = 1 << d.logN;
    const int lt = int(threadIdx.x);
    const int i = rb0 >> logN1;
    const int u0 = rb0 & ((1 << logN1) - 1), u1 = rb1 & ((1 << logN1) - 1);
    const uint32_t p = __ldg(&t.pc32[i].p), pinv = __ldg(&t.pc32[i].pinv);
    uint32_t* buf = reinterpret_cast<uint32_t*>(smem);
    uint32_t* buf_a = buf + S::N2;
    uint2* const s_tw0 = reinterpret_cast<uint2*>(smem + size_t(2) * S::N2 * 4);
    uint2* const s_tw1 = s_tw0 + S::N2;
    const uint2* twf = t.fwd32 + size_t(i) * kMaxN;
    const uint32_t* ra = reinterpret_cast<const uint32_t*>(d.ra);
    const uint32_t* rbr = reinterpret_cast<const uint32_t*>(d.rb);
    uint32_t* out = reinterpret_cast<uint32_t*>(d.ra);
    const size_t off0 = size_t(i) * N + size_t(u0) * S::N2, off1 = size_t(i) * N + size_t(u1) * S::N2;
    // lt 0: one arrival expecting the block of a of the member at `off`, and its copy
    auto copy_blocks = [&](size_t off) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(4u * S::N2) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(buf_a)),
                     "l"(ra + off), "r"(4u * S::N2), "r"(bar)
                     : "memory");
    };
    // the same block by plain loads, every thread
    auto load_blocks = [&](size_t off) {
        for (int x = lt; x < S::N2; x += S::T) buf_a[x] = __ldcg(ra + off + x);
    };

    __syncthreads();  // shared memory of a previous item is free
    if (use_bulk && lt == 0) {
        // the twiddles do not depend on the previous kernel: their copies start before its end
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(16u * ((1u << LOG_N2) - 2u))
                     : "memory");
        stage_twiddles<LOG_N2>(twf, (1 << logN1) + u0, s_tw0, bar);
        stage_twiddles<LOG_N2>(twf, (1 << logN1) + u1, s_tw1, bar);
    }
    pdl_wait();  // the residues come from the stream's previous kernel
    if (use_bulk && lt == 0) {
        asm volatile("fence.proxy.async.global;" ::: "memory");  // the previous kernel's writes -> bulk reads
        copy_blocks(off0);
    }
    // phase whose copies may still be in flight (-1: none) once a wait gave up
    int pending = -1;
    bool staged = use_bulk && __syncthreads_and(bar_wait(bar, parity) ? 1 : 0) != 0;
    if (!staged) {
        if (use_bulk) pending = 0;
        copy_twiddles<LOG_N2>(twf, (1 << logN1) + u0, s_tw0, lt, S::T);
        copy_twiddles<LOG_N2>(twf, (1 << logN1) + u1, s_tw1, lt, S::T);
        load_blocks(off0);
        __syncthreads();
    }
    const uint32_t p2 = 2 * p;
#pragma unroll 1
    for (int j = 0; j < 2; ++j) {
        const size_t off = j ? off1 : off0;
        if (j == 1) {
            if (staged) {
                staged = __syncthreads_and(bar_wait(bar, parity ^ 1u) ? 1 : 0) != 0;
                if (!staged) pending = 1;
            } else if (pending == 0) {
                // once the late copies of the first member are done, its buffers are free
                if (__syncthreads_and(bar_wait(bar, parity) ? 1 : 0) != 0)
                    pending = -1;
                else if (error && lt == 0 && atomicCAS(error, 0u, 1u) == 0u)
                    error[1] = what;
            }
            if (!staged) {
                load_blocks(off1);
                __syncthreads();
            }
        }
        uint32_t v[S::E];
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = buf_a[row_index<S, 0>(lt, e)];
        if constexpr (S::NPASS == 1) __syncthreads();  // buf_a's raw block is read before it is rewritten
        row_forward_from<S, 0>(v, buf, j ? s_tw1 : s_tw0, lt, p);
        row_store<S, LAST>(v, buf_a, lt);
#pragma unroll
        for (int e = 0; e < S::E; ++e) v[e] = __ldcg(rbr + off + row_index<S, 0>(lt, e));
        row_forward_from<S, 0>(v, buf, j ? s_tw1 : s_tw0, lt, p);
        __syncthreads();
        {
            uint32_t av[S::E];
            row_load<S, LAST>(av, buf_a, lt);
#pragma unroll
            for (int e = 0; e < S::E; ++e) v[e] = mont(csub(csub(av[e], p2), p), v[e], p, pinv);
        }
        if (j == 0) {
            __syncthreads();  // every thread has read buf_a
            if (staged && lt == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // those reads -> the bulk writes
                copy_blocks(off1);
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
            }
        }
        row_inverse_from<S, LAST>(v, buf, j ? s_tw0 : s_tw1, lt, p);
#pragma unroll
        for (int e = 0; e < S::E; ++e) __stcg(out + off + row_index<S, 0>(lt, e), v[e]);
    }
    if (pending >= 0) bar_wait(bar, pending ? parity ^ 1u : parity);  // copies in flight end before the smem is reused
    return use_bulk && pending < 0;
}

}  // namespace w32

}  // namespace nc
