// Kernels of the 30-bit word engine (w32.cuh): k_dec_tc32 (residues on the tensor cores + forward
// column stages), k_row32 (row blocks) and k_crt_tc32 (inverse column stages + CRT on the tensor
// cores + Barrett), with their launchers.
//
// Residues. With x_n given as 4 L bytes x_{n,b}, x_n mod p_i = sum_c 2^(8 c) S[n][i,c] with
// S[n][i,c] = sum_b x_{n,b} w_{i,b,c}, w_{i,b,c} byte c (of 4) of 2^(8 b) mod p_i: the same u8 x u8
// contraction as the 62-bit engine's k_dec_tc, with four byte planes a prime instead of eight, so
// one pass of MMAs (128 accumulator columns) covers 32 primes. The folded sum (< 2^48) is reduced
// with one multiply by floor(2^50 / p).
//
// CRT. v_i = r_i y_i mod p_i < 2^30 is 4 bytes, so A has K = 4 k <= 256 bytes and the table B has
// B[c][4 i + a] = byte c - a of (M/p_i) mod q; every S_c < 4 k 255^2 < 2^24.
#include "batch_types.h"
#include "crt_tc.cuh"
#include "kernel_registry.h"
#include "w32.cuh"

namespace nc {

namespace w32 {

namespace {

using crt_tc_detail::a_offset;
using crt_tc_detail::kmajor_desc;
using crt_tc_detail::mma_wait;
using crt_tc_detail::smem_u32;

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ uint64_t mad_wide(uint32_t a, uint32_t b, uint64_t c) {
    uint64_t d;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
    return d;
}

// sum_c 2^(8 c) s[c] mod p into [0, 2p), for s[c] < 2^23 (so the sum V < 2^48) and p in
// (2^29, 2^30): with A = V >> 28 and bar = floor(2^50 / p), floor(A bar / 2^22) falls short of
// V / p by less than 2^28 / p + 2^20 / 2^22 < 0.75, so it is floor(V / p) or one less.
__device__ __forceinline__ uint32_t fold_planes(const uint32_t* s, uint32_t p, uint32_t bar) {
    const uint64_t v = mad_wide(s[3], 1u << 24, mad_wide(s[2], 1u << 16, mad_wide(s[1], 1u << 8, uint64_t(s[0]))));
    const uint32_t qh = uint32_t((uint64_t(uint32_t(v >> 28)) * bar) >> 22);
    return uint32_t(v) - qh * p;
}

// Residue row of prime i (128 u32) over its pair's 1 KB of weights.
__device__ __forceinline__ uint32_t* res_row(uint8_t* sB, int i) { return reinterpret_cast<uint32_t*>(sB + i * 512); }

// Slot of tile row x in prime i's residue row. Every prime's row starts on bank 0, so rows are
// XORed (bits 2-4 for 4-column tiles, bits 0-4 otherwise) by the prime and, for 4-column tiles,
// by the half of the 32-point column (bit 5): the column stages' loads of one warp then fall on
// 32 different banks, and the fold's stores (32 consecutive rows) stay conflict-free.
__device__ __forceinline__ int res_slot(int i, int x, int C) {
    const int f = C == 4 ? ((((i & 3) << 1) | ((x >> 5) & 1)) << 2) : ((i * C) & 31);
    return x ^ f;
}

// Weight pairs a launch copies: the primes rounded up to a multiple of four (an MMA's N is a
// multiple of 16 columns), within the table's 64 primes.
__host__ __device__ constexpr int dec32_weight_pairs(int k) { return ((k + 3) & ~3) / 2; }

// CC: the tile's columns when N >= 128 (128 >> LOG_N1, a constant: the index arithmetic of the
// fold and the column stages folds away), 0 for smaller N.
template <int LOG_N1, int CC>
__device__ __forceinline__ void dec_tc32_item(const ProductDesc& d, const Tables& t, int operand, int tile,
                                              uint8_t* smem, uint64_t& bar, uint32_t& taddr_slot) {
    constexpr int N1 = 1 << LOG_N1;
    const int N = 1 << d.logN;
    const int N2 = N >> LOG_N1;
    const int T = CC ? kDecTcRows : (N < kDecTcRows ? N : kDecTcRows);
    const int logC = CC ? 7 - LOG_N1 : (N < kDecTcRows ? int(d.logN) : 7) - LOG_N1;
    const int C = CC ? CC : 1 << logC;
    const int j0 = tile * C;
    const int L = int(d.L), k = int(d.k);
    const int wpairs = dec32_weight_pairs(k);
    const uint32_t* x = factor_limbs(d, operand);
    uint32_t* R = reinterpret_cast<uint32_t*>(factor_residues(d, operand));
    uint8_t* sA = smem;                     // [16 row groups][8 K chunks][8 rows][16 B]
    uint8_t* sB = smem + kDecTcRows * 128;  // [prime pair][8 K chunks][8 rows][16 B]
    PrimeConst32* s_pc = reinterpret_cast<PrimeConst32*>(sB + wpairs * 1024);
    const int tid = int(threadIdx.x), warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&taddr_slot)),
                     "r"(kDecTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // dependents are released only once every CTA holds its tensor memory (as in k_dec_tc)
    __syncthreads();
    pdl_trigger();

    for (int q = tid; q < wpairs * 64; q += kThreads) cp_async16(sB + q * 16, t.res_w32 + q);
    for (int w = tid; w < ((k + 3) & ~3); w += kThreads) s_pc[w] = t.pc32[w];  // the MMAs' primes
    pdl_wait();  // the operand and the residue rows belong to the stream's previous kernels
    const int kbytes = 4 * L;
    for (int q = tid; q < kDecTcRows * 8; q += kThreads) {
        const int rlo = q & 7, kc = (q >> 3) & 7, rg = q >> 6;
        const int m = rg * 8 + rlo;
        uint8_t* dst = sA + rg * 1024 + kc * 128 + rlo * 16;
        if (m < T && kc * 16 < kbytes) {
            const int n = (m >> logC) * N2 + j0 + (m & (C - 1));
            const uint32_t* row = x + size_t(n) * size_t(L);
            const int l0 = kc * 4;
            if ((L & 3) == 0) {
                cp_async16(dst, row + l0);
            } else if ((L & 1) == 0) {
                cp_async8(dst, row + l0, 8u);
                cp_async8(dst + 8, l0 + 2 < L ? row + l0 + 2 : row, l0 + 2 < L ? 8u : 0u);
            } else {
#pragma unroll
                for (int w = 0; w < 4; ++w) cp_async4(dst + 4 * w, l0 + w < L ? row + l0 + w : row, l0 + w < L ? 4u : 0u);
            }
        } else {
            *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = taddr_slot;
    const int slices = (kbytes + 31) / 32;

    // passes of 32 primes; warp w reads tensor-memory lanes 32 (w % 4) .. and half w / 4 of the
    // pass's primes (16 of them, four per 16-column load)
    const int m = 32 * (warp & 3) + lane;
    const int half = warp >> 2;
    bool failed = false;
    for (int g = 0; g * kDecTc32PassPrimes < k; ++g) {
        const int i0 = g * kDecTc32PassPrimes;
        const int np = k - i0 < kDecTc32PassPrimes ? k - i0 : kDecTc32PassPrimes;
        if (tid == 0 && !failed) {
            const uint32_t ncols = uint32_t(((np + 3) & ~3) * 4);
            const uint32_t idesc = (2u << 4) | ((ncols >> 3) << 17) | (uint32_t(kDecTcRows >> 4) << 24);
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB + (i0 >> 1) * 1024);
            for (int s = 0; s < slices; ++s) {
                const uint64_t da = kmajor_desc(a0 + uint32_t(s) * 256u, 128u, 1024u);
                const uint64_t db = kmajor_desc(b0 + uint32_t(s) * 256u, 128u, 1024u);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
                    "l"(da), "l"(db), "r"(idesc), "r"(s));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bar))
                         : "memory");
        }
        const bool ok = !failed && mma_wait(smem_u32(&bar), uint32_t(g & 1));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int ib = i0 + 16 * half;
        const int ie = i0 + np < ib + 16 ? i0 + np : ib + 16;
        if (__all_sync(0xffffffffu, ok)) {
            const uint32_t lane_base = taddr + (uint32_t(32 * (warp & 3)) << 16);
            for (int i = ib; i < ie; i += 4) {
                uint32_t s[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]),
                      "=r"(s[8]), "=r"(s[9]), "=r"(s[10]), "=r"(s[11]), "=r"(s[12]), "=r"(s[13]), "=r"(s[14]),
                      "=r"(s[15])
                    : "r"(lane_base + uint32_t(4 * (i - i0))));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                // all four (primes up to k rounded up to four have weights, constants and rows)
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    res_row(sB, i + e)[res_slot(i + e, m, C)] = fold_planes(s + 4 * e, s_pc[i + e].p, s_pc[i + e].bar);
            }
        } else if (m < T) {
            // the wait gave up: this warp's residues on the integer pipes
            const int n = (m >> logC) * N2 + j0 + (m & (C - 1));
            const uint32_t* row = x + size_t(n) * size_t(L);
            for (int i = ib; i < ie; ++i) {
                const uint64_t p = s_pc[i].p;
                uint64_t acc = 0;
                for (int l = 0; l < L; ++l)
                    acc = (acc + uint64_t(__ldg(row + l)) * __ldg(t.pow32_32 + size_t(i) * kMaxL + l)) % p;
                res_row(sB, i)[res_slot(i, m, C)] = uint32_t(acc);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        failed = __syncthreads_or(ok ? 0 : 1) != 0;  // also: this pass's reads are done before the next MMA
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kDecTcCols) : "memory");

    // forward column stages of items (prime i, column j), then the residue rows
    if constexpr (LOG_N1 == 5) {
        // 32-point columns on two adjacent lanes, as in k_dec_tc: lane h runs the first stage's
        // butterflies (u, u + 16) for u in [8h, 8h + 8), the lanes swap halves, and each runs the
        // four remaining stages on its half-subtree (twiddle root 2 + h)
        const int total = 2 * k * C;
        for (int w0 = tid & ~31; w0 < total; w0 += kThreads) {
            const int w = w0 + lane;
            const bool active = w < total;
            const int item = active ? w >> 1 : 0, h = w & 1;
            const int i = item >> logC, j = item & (C - 1);
            const uint32_t* sr = res_row(sB, i);
            const uint32_t p = s_pc[i].p, p2 = 2 * p;
            const uint2* tw = t.fwd32 + size_t(i) * kMaxN;
            uint32_t xs[8], ys[8];
            const uint2 w1 = __ldg(tw + 1);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int u = 8 * h + e;
                xs[e] = sr[res_slot(i, u * C + j, C)];
                ys[e] = sr[res_slot(i, (u + 16) * C + j, C)];
                w32::ct_bfly(xs[e], ys[e], w1.x, w1.y, p, p2);
            }
            uint32_t v[16];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint32_t got = __shfl_xor_sync(0xffffffffu, h ? xs[e] : ys[e], 1);
                v[e] = h ? got : xs[e];
                v[8 + e] = h ? ys[e] : got;
            }
            w32::column_forward_root<4>(tw, 2 + h, p, v);
            if (active) {
                uint32_t* out = R + size_t(i) * N + j0 + j + size_t(16 * h) * N2;
#pragma unroll
                for (int u = 0; u < 16; ++u) __stcg(out + size_t(u) * N2, v[u]);
            }
        }
    } else {
        for (int w = tid; w < k * C; w += kThreads) {
            const int i = w >> logC, j = w & (C - 1);
            const uint32_t* sr = res_row(sB, i);
            uint32_t v[N1];
#pragma unroll
            for (int u = 0; u < N1; ++u) v[u] = sr[res_slot(i, u * C + j, C)];
            if (LOG_N1 > 0) w32::column_forward_root<LOG_N1>(t.fwd32 + size_t(i) * kMaxN, 1, s_pc[i].p, v);
            uint32_t* out = R + size_t(i) * N + j0 + j;
#pragma unroll
            for (int u = 0; u < N1; ++u) __stcg(out + size_t(u) * N2, v[u]);
        }
    }
}

// Four CTAs per SM, as k_dec_tc (tensor memory holds four of 128 columns).
template <int LOG_N1>
__global__ void __launch_bounds__(kThreads, 4) k_dec_tc32(ProductDesc d, Tables t, int first_operand, int tile0,
                                                           int tiles) {
#if NC_HAS_TCGEN05
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    const int operand = first_operand + int(blockIdx.x) / tiles, tile = tile0 + int(blockIdx.x) % tiles;
    if (d.logN >= 7)
        dec_tc32_item<LOG_N1, (kDecTcRows >> LOG_N1)>(d, t, operand, tile, smem, bar, taddr_slot);
    else
        dec_tc32_item<LOG_N1, 0>(d, t, operand, tile, smem, bar, taddr_slot);
#endif
}

// ------------------------------------------------------------------------------------------
// CRT: inverse column stages, v_i = r_i y_i mod p_i into A (4 bytes at K offset 4 i), the
// contraction, the quotient estimate and Barrett (crt_coeffs_tc of crt_tc.cuh on 30-bit residues)

template <int LOG_N1>
__device__ void crt32_columns(const ProductDesc& d, const Tables& t, int j0, int T, const uint32_t* s_y,
                              const uint32_t* s_ys, const uint32_t* s_p, uint8_t* sA) {
    constexpr int N1 = 1 << LOG_N1;
    const int N = 1 << d.logN;
    const int N2 = N >> LOG_N1;
    const int C = T >> LOG_N1;
    const int k = int(d.k);
    const uint32_t* res = reinterpret_cast<const uint32_t*>(d.ra);
    auto put = [&](int tc, int i, uint32_t v) {
        *reinterpret_cast<uint32_t*>(sA + (tc >> 7) * kCrtTcHalfBytes + a_offset(tc & 127, 4 * i)) = v;
    };
    if constexpr (LOG_N1 == 5) {
        // 32-point columns on two adjacent lanes (as crt_columns_tc): lane h loads rows
        // [16h, 16h + 16), runs the inverse stages of its half-subtree, and the last stage's pairs
        // (u, u + 16) are split between the lanes after one exchange of eight values
        const int total = 2 * k * C;
        const int lane = int(threadIdx.x) & 31;
        for (int w0 = int(threadIdx.x) & ~31; w0 < total; w0 += int(blockDim.x)) {
            const int w = w0 + lane;
            const bool active = w < total;
            const int item = active ? w >> 1 : 0, h = w & 1;
            const int i = item / C, j = item - i * C;
            const uint32_t* row = res + size_t(i) * N + j0 + j + size_t(16 * h) * N2;
            uint32_t v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = active ? __ldcg(row + size_t(u) * N2) : 0u;
            const uint32_t p = s_p[i], p2 = 2 * p;
            const uint2* tw = t.inv32 + size_t(i) * kMaxN;
            w32::column_inverse_root<4>(tw, 2 + h, p, v);
            const uint2 w1 = __ldg(tw + 1);
            const uint32_t y = s_y[i], ys = s_ys[i];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint32_t got = __shfl_xor_sync(0xffffffffu, h ? v[e] : v[8 + e], 1);
                uint32_t lo = h ? got : v[e], hi = h ? v[8 + e] : got;  // rows 8h + e and 8h + e + 16
                w32::gs_bfly(lo, hi, w1.x, w1.y, p, p2);
                if (active) {
                    put((8 * h + e) * C + j, i, w32::csub(w32::shoup(lo, y, ys, p), p));
                    put((8 * h + e + 16) * C + j, i, w32::csub(w32::shoup(hi, y, ys, p), p));
                }
            }
        }
    } else {
        for (int w = threadIdx.x; w < k * C; w += blockDim.x) {
            const int i = w / C, j = w - i * C;
            const uint32_t* row = res + size_t(i) * N + j0 + j;
            uint32_t v[N1];
#pragma unroll
            for (int u = 0; u < N1; ++u) v[u] = __ldcg(row + size_t(u) * N2);
            const uint32_t p = s_p[i];
            if (LOG_N1 > 0) w32::column_inverse_root<LOG_N1>(t.inv32 + size_t(i) * kMaxN, 1, p, v);
            const uint32_t y = s_y[i], ys = s_ys[i];
#pragma unroll
            for (int u = 0; u < N1; ++u) put(u * C + j, i, w32::csub(w32::shoup(v[u], y, ys, p), p));
        }
    }
}

// Shared memory of the 30-bit CRT: A (two halves of 128 rows x 256 K bytes), the plan's table,
// y, its companion and p of up to 64 primes, (-M) mod q, q and mu; raised so that no more CTAs
// share an SM than its tensor memory holds (as crt_tc_smem_bytes).
NC_HD constexpr size_t crt_tc32_smem_bytes(int LW) {
    return smax(size_t(2) * kCrtTcHalfBytes + crt_tc_table_bytes(LW) + size_t(kMaxPrimes32) * 4 * 3 +
                    size_t(kMqStride) * 4 * 2 + 16 + 16,
                (size_t(233472) / (512 / crt_tc_tmem_cols(LW) + 1) + 16) / 16 * 16);
}

template <int LW>
__device__ void crt32_coeffs_tc(const ProductDesc& d, const Tables& t, int tile, uint8_t* smem, uint32_t taddr,
                                uint64_t* bar, uint32_t parity) {
    constexpr int W = LW + kAccExtra;
    constexpr int NC = crt_tc_cols(LW);
    constexpr uint32_t kHalfCol = crt_tc_tmem_cols(LW) / 2;
    const int N = 1 << d.logN;
    const int logN1 = int(d.logN) - int(d.logN2);
    const int N2 = N >> logN1;
    const int T = N < kTile ? N : kTile;
    const int C = T >> logN1;
    const int k = int(d.k), L = int(d.L);
    const int j0 = tile * C;

    uint8_t* sA = smem;
    uint8_t* sB = smem + 2 * kCrtTcHalfBytes;
    uint32_t* s_y = reinterpret_cast<uint32_t*>(sB + NC * 256);
    uint32_t* s_ys = s_y + kMaxPrimes32;
    uint32_t* s_p = s_ys + kMaxPrimes32;
    uint32_t* s_negm = s_p + kMaxPrimes32;
    uint32_t* s_q = s_negm + kMqStride;
    uint32_t* s_mu = s_q + kMqStride;
    const int tid = int(threadIdx.x), warp = tid >> 5;

    __syncthreads();
    const QConst32* qc = d.qc32;
    for (int w = tid; w < k; w += blockDim.x) {
        s_y[w] = __ldg(qc->y + w);
        s_ys[w] = __ldg(qc->ys + w);
        s_p[w] = __ldg(&t.pc32[w].p);
    }
    for (int w = tid; w < kMqStride; w += blockDim.x) {
        s_negm[w] = __ldg(qc->neg_m + w);
        s_q[w] = __ldg(qc->q + w);
    }
    if (tid < 4) s_mu[tid] = __ldg(qc->mu + tid);
    // the table is first read by the MMAs: its copy runs behind the column stages (its K bytes
    // from 4 k up to the last slice's end are zero, so A's are never read into the sums)
    for (int w = tid; w < NC * 16; w += blockDim.x) cp_async16(sB + 16 * w, d.crt_b + w);
    asm volatile("cp.async.commit_group;" ::: "memory");
    __syncthreads();
    pdl_wait();  // the residues come from the stream's previous kernel

    switch (logN1) {
        case 0: crt32_columns<0>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 1: crt32_columns<1>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 2: crt32_columns<2>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 3: crt32_columns<3>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 4: crt32_columns<4>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        default: crt32_columns<5>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (tid == 0) {
        const uint32_t idesc = (2u << 4) | (uint32_t(NC >> 3) << 17) | (uint32_t(128 >> 4) << 24);
        const int slices = (4 * k + 31) / 32;
        const uint32_t b0 = smem_u32(sB);
        for (int h = 0; h < (T > 128 ? 2 : 1); ++h) {
            const uint32_t a0 = smem_u32(sA + h * kCrtTcHalfBytes);
            for (int s = 0; s < slices; ++s) {
                const uint64_t da = kmajor_desc(a0 + uint32_t(s) * 256u, 128u, 2048u);
                const uint64_t db = kmajor_desc(b0 + uint32_t(s) * 256u, 128u, 2048u);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr + uint32_t(h) * kHalfCol),
                    "l"(da), "l"(db), "r"(idesc), "r"(s));
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                     : "memory");
    }

    // while the MMAs run: this thread's coefficient and the CRT quotient round(sum v_i / p_i)
    const int tc = tid;
    const int half = tc >> 7;
    const uint8_t* arow = sA + half * kCrtTcHalfBytes + a_offset(tc & 127, 0);
    uint64_t frac = 0;
#pragma unroll 4
    for (int i = 0; i < k; ++i) {
        const uint32_t v = *reinterpret_cast<const uint32_t*>(arow + (i >> 2) * 128 + (i & 3) * 4);
        frac += (uint64_t(v) * __ldg(&t.pc32[i].quo)) >> 29;  // 2^32 v / p_i, short by less than 3
    }
    const uint32_t kq = uint32_t((frac + (1ull << 31)) >> 32);

    const bool ok = mma_wait(smem_u32(bar), parity);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    uint32_t acc[W];
#pragma unroll
    for (int w = 0; w < W; ++w) acc[w] = 0;
    if (__all_sync(0xffffffffu, ok)) {
        const uint32_t lane_base = taddr + (uint32_t(32 * (warp & 3)) << 16) + uint32_t(half) * kHalfCol;
        uint64_t carry = 0;
#pragma unroll
        for (int cb = 0; cb < NC / 8; ++cb) {
            uint32_t s[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7])
                : "r"(lane_base + uint32_t(8 * cb)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const uint64_t t0 = carry + s[0] + (uint64_t(s[1]) << 8) + (uint64_t(s[2]) << 16) + (uint64_t(s[3]) << 24);
            if (2 * cb < W) acc[2 * cb] = uint32_t(t0);
            const uint64_t t1 =
                (t0 >> 32) + s[4] + (uint64_t(s[5]) << 8) + (uint64_t(s[6]) << 16) + (uint64_t(s[7]) << 24);
            if (2 * cb + 1 < W) acc[2 * cb + 1] = uint32_t(t1);
            carry = t1 >> 32;
        }
    } else {
        // the MMAs did not report completion in time: the same sum on the integer pipes
        uint32_t acc_hi[W];
#pragma unroll
        for (int w = 0; w < W; ++w) acc_hi[w] = 0;
#pragma unroll 1
        for (int i = 0; i < k; ++i) {
            const uint32_t v = *reinterpret_cast<const uint32_t*>(arow + (i >> 2) * 128 + (i & 3) * 4);
            const uint32_t* M = qc->mq + i * kMqStride;
            uint32_t m[LW];
#pragma unroll
            for (int l = 0; l < LW; ++l) m[l] = __ldg(M + l);
            mac_lo<LW, 0, W>(acc, m, v);
            mac_hi<LW, 1, W>(acc_hi, m, v);
        }
        asm volatile("add.cc.u32 %0, %0, %1;" : "+r"(acc[0]) : "r"(acc_hi[0]));
#pragma unroll
        for (int w = 1; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, %1;" : "+r"(acc[w]) : "r"(acc_hi[w]));
        asm volatile("addc.u32 %0, %0, %1;" : "+r"(acc[W - 1]) : "r"(acc_hi[W - 1]));
    }
    {
        uint32_t acc_hi[W];
#pragma unroll
        for (int w = 0; w < W; ++w) acc_hi[w] = 0;
        mac_lo<LW, 0, W>(acc, s_negm, kq);
        mac_hi<LW, 1, W>(acc_hi, s_negm, kq);
        asm volatile("add.cc.u32 %0, %0, %1;" : "+r"(acc[0]) : "r"(acc_hi[0]));
#pragma unroll
        for (int w = 1; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, %1;" : "+r"(acc[w]) : "r"(acc_hi[w]));
        asm volatile("addc.u32 %0, %0, %1;" : "+r"(acc[W - 1]) : "r"(acc_hi[W - 1]));
    }
    uint32_t r[LW + 1];
    barrett<LW, W>(acc, s_q, s_mu, int(qc->qbits), r);

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    uint32_t* s_out = reinterpret_cast<uint32_t*>(sA);
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

template <int LW>
__global__ void __launch_bounds__(kThreads, 2) k_crt_tc32(ProductDesc d, Tables t) {
#if NC_HAS_TCGEN05
    constexpr uint32_t kCols = crt_tc_tmem_cols(LW);
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&taddr_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    pdl_trigger();  // only once the CTA holds its tensor memory
    const uint32_t taddr = taddr_slot;
    crt32_coeffs_tc<LW>(d, t, int(blockIdx.x), smem, taddr, &bar, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kCols) : "memory");
#endif
}

// ------------------------------------------------------------------------------------------
// row blocks

// Resident CTAs per SM: radix-8 passes in 256-thread CTAs at four (64 registers; at N = 2^16,
// k = 59: 40.0 us, against 39.9 at three and 40.9 at five), radix 16 at three.
template <int LOG_N2, int LOG_E, int THREADS>
__global__ void __launch_bounds__(THREADS, (THREADS == 256 ? (LOG_E == 3 ? 4 : 3) : 2)) k_row32(ProductDesc d, Tables t) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    pdl_trigger();
    const uint32_t b = smem_u32(&bar);
    w32::row_barrier_init<LOG_N2, LOG_E, THREADS>(b);
    w32::row_blocks<LOG_N2, LOG_E, THREADS>(d, t, int(blockIdx.x), smem, b, 0, true);
}

#define NC_ROW32_VARIANTS(X)                                                                                   \
    X(1, 4, 256) X(2, 4, 256) X(3, 4, 256) X(4, 4, 256) X(5, 4, 256) X(6, 4, 256) X(7, 4, 256) X(8, 4, 256)  \
    X(9, 4, 256) X(10, 4, 256) X(11, 4, 256) X(12, 4, 256) X(6, 3, 256) X(7, 3, 256) X(8, 3, 256)           \
    X(9, 3, 256) X(10, 3, 256) X(11, 3, 256) X(12, 3, 512)

// ------------------------------------------------------------------------------------------
// batches (products of N < 2^15 on the 30-bit engine; batch.cu): the residue items of every such
// product (one CTA per item), then one persistent row launch per row-block size, then the CRT
// items. The launches of a batch run in stream order, so no item waits on another.

// Residue items (x = product, y = operand * tiles_tc + tile), every product of the launch with
// column length 2^LOG_N1.
template <int LOG_N1>
__global__ void __launch_bounds__(kThreads, 4) k_batch_dec_tc32(BatchCrtArgs a) {
#if NC_HAS_TCGEN05
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    const uint2 w = __ldg(a.items + blockIdx.x);
    const BatchProduct& bp = a.products[w.x];
    const int tiles = int(bp.tiles_tc);
    const int operand = int(bp.first_operand) + int(w.y) / tiles, tile = int(w.y) % tiles;
    if (bp.d.logN >= 7)
        dec_tc32_item<LOG_N1, (kDecTcRows >> LOG_N1)>(bp.d, a.tables, operand, tile, smem, bar, taddr_slot);
    else
        dec_tc32_item<LOG_N1, 0>(bp.d, a.tables, operand, tile, smem, bar, taddr_slot);
#endif
}

// Row items (x = product, y = row-CTA index) with row blocks of 2^LOG_N2, radix 8, 256 threads:
// persistent CTAs take items in queue order; each item's twiddles and residue blocks arrive on the
// CTA's mbarrier, one phase per item. If a bulk wait gives up (the item then loads its data with
// plain loads), the CTA's later items use plain loads too.
template <int LOG_N2>
__global__ void __launch_bounds__(kThreads, 4) k_persistent_rows32(BatchArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ int s_item;
    __shared__ __align__(16) BatchProduct s_bp;
    constexpr int kWords = int(sizeof(BatchProduct) / 4);
    // with one row block a CTA, items come two at a time: a mirror pair (adjacent in the queue,
    // batch.cu) runs as row_pair, anything else as two row_blocks
    constexpr bool kPairs = RowShape<LOG_N2, kBatchRowLogE>::T == kThreads;
    pdl_trigger();
    const uint32_t b = smem_u32(&bar);
    row_barrier_init<LOG_N2, kBatchRowLogE, kThreads>(b);
    uint32_t parity = 0;
    bool bulk = true;
    auto load_product = [&](uint32_t x) {
        if (threadIdx.x < kWords)
            reinterpret_cast<uint32_t*>(&s_bp)[threadIdx.x] =
                __ldg(reinterpret_cast<const uint32_t*>(a.products + (x & 0x0fffffffu)) + threadIdx.x);
        __syncthreads();
    };
    auto single = [&](int y) {
        const bool ok = row_blocks<LOG_N2, kBatchRowLogE, kThreads>(s_bp.d, a.tables, y, smem, b, parity, bulk);
        if (bulk) parity ^= 1u;
        bulk = bulk && ok;  // the item's result stands either way; later items avoid the barrier
    };
    for (;;) {
        if (threadIdx.x == 0) s_item = int(atomicAdd(a.head, kPairs ? 2u : 1u));
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const uint2 w = __ldg(a.items + it);
        load_product(w.x);
        if constexpr (kPairs) {
            const bool has2 = it + 1 < a.n_items;
            const uint2 w2 = has2 ? __ldg(a.items + it + 1) : make_uint2(0u, 0u);
            const int logN1 = int(s_bp.d.logN) - LOG_N2;
            const int mask = (1 << logN1) - 1;
            const int mirror = (int(w.y) & ~mask) | (mask - (int(w.y) & mask));
            if (has2 && w2.x == w.x && s_bp.d.mode == kModeProduct && logN1 >= 1 && int(w2.y) == mirror) {
                // two phases when the copies ran, so the parity is unchanged
                bulk = row_pair<LOG_N2, kBatchRowLogE, kThreads>(s_bp.d, a.tables, int(w.y), int(w2.y), smem, b, parity,
                                                                 bulk, a.error, w.x);
            } else {
                single(int(w.y));
                if (has2) {
                    __syncthreads();  // s_bp is rewritten
                    load_product(w2.x);
                    single(int(w2.y));
                }
            }
        } else {
            single(int(w.y));
        }
        __syncthreads();  // s_item and s_bp are rewritten by the next round
    }
}

// CRT items (x = product, y = 256-coefficient tile); products of at most 30 limbs (256 columns of
// tensor memory per CTA).
__global__ void __launch_bounds__(kThreads, 2) k_batch_crt_tc32(BatchCrtArgs a) {
#if NC_HAS_TCGEN05
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(&taddr_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    pdl_trigger();  // only once the CTA holds its tensor memory
    const uint32_t taddr = taddr_slot;
    const uint2 w = __ldg(a.items + blockIdx.x);
    const BatchProduct& bp = a.products[w.x];
    switch (bp.d.LW) {
#define NC_B_CRT_TC32(n)                                                        \
    case n:                                                                     \
        if constexpr (crt_tc_tmem_cols(n) == 256)                               \
            crt32_coeffs_tc<n>(bp.d, a.tables, int(w.y), smem, taddr, &bar, 0); \
        break;
        NC_LW_CASES(NC_B_CRT_TC32)
#undef NC_B_CRT_TC32
        default: break;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(taddr) : "memory");
#endif
}

void* batch_dec_tc32_kernel(int logN1) {
    switch (logN1) {
        case 0: return reinterpret_cast<void*>(&k_batch_dec_tc32<0>);
        case 1: return reinterpret_cast<void*>(&k_batch_dec_tc32<1>);
        case 2: return reinterpret_cast<void*>(&k_batch_dec_tc32<2>);
        case 3: return reinterpret_cast<void*>(&k_batch_dec_tc32<3>);
        case 4: return reinterpret_cast<void*>(&k_batch_dec_tc32<4>);
        case 5: return reinterpret_cast<void*>(&k_batch_dec_tc32<5>);
        default: return nullptr;
    }
}

void* persistent_rows32_kernel(int logN2) {
    switch (logN2) {
#define NC_P_ROWS32(n) \
    case n: return reinterpret_cast<void*>(&k_persistent_rows32<n>);
        NC_P_ROWS32(1) NC_P_ROWS32(2) NC_P_ROWS32(3) NC_P_ROWS32(4) NC_P_ROWS32(5) NC_P_ROWS32(6)
        NC_P_ROWS32(7) NC_P_ROWS32(8) NC_P_ROWS32(9) NC_P_ROWS32(10) NC_P_ROWS32(11)
#undef NC_P_ROWS32
        default: return nullptr;
    }
}

void* dec_tc32_kernel(int logN1) {
    switch (logN1) {
        case 0: return reinterpret_cast<void*>(&k_dec_tc32<0>);
        case 1: return reinterpret_cast<void*>(&k_dec_tc32<1>);
        case 2: return reinterpret_cast<void*>(&k_dec_tc32<2>);
        case 3: return reinterpret_cast<void*>(&k_dec_tc32<3>);
        case 4: return reinterpret_cast<void*>(&k_dec_tc32<4>);
        case 5: return reinterpret_cast<void*>(&k_dec_tc32<5>);
        default: return nullptr;
    }
}

void* crt_tc32_kernel(int LW) {
    switch (LW) {
#define NC_CRT_TC32(n) \
    case n: return reinterpret_cast<void*>(&k_crt_tc32<n>);
        NC_LW_CASES(NC_CRT_TC32)
#undef NC_CRT_TC32
        default: return nullptr;
    }
}

}  // namespace

}  // namespace w32

// Shared memory of the 30-bit residue stage: the limb tile, the weights of the primes it
// copies and their constants; raised, as dec_tc_smem_bytes, to keep four CTAs per SM.
size_t dec_tc32_smem_bytes(int k) {
    return smax(size_t(kDecTcRows) * 128 + size_t(w32::dec32_weight_pairs(k)) * 1024 + size_t(kMaxPrimes32) * 16,
                (size_t(233472) / (512 / kDecTcCols + 1) + 16) / 16 * 16);
}

void* row32_kernel(const RowConfig& c) {
#define NC_ROW32(n, e, th) \
    if (c.logN2 == n && c.logE == e && c.threads == th) return reinterpret_cast<void*>(&w32::k_row32<n, e, th>);
    NC_ROW32_VARIANTS(NC_ROW32)
#undef NC_ROW32
    return nullptr;
}

std::vector<RowConfig> all_row32_variants() {
    std::vector<RowConfig> v;
#define NC_ROW32_LIST(n, e, th) v.push_back(RowConfig{n, e, th});
    NC_ROW32_VARIANTS(NC_ROW32_LIST)
#undef NC_ROW32_LIST
    return v;
}

cudaError_t prepare_w32() {
    cudaError_t e = cudaSuccess;
    for (const RowConfig& c : all_row32_variants()) {
        if (e != cudaSuccess) break;
        e = cudaFuncSetAttribute(row32_kernel(c), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(w32::row_smem_bytes(c.threads, c.logE)));
    }
    for (int l = 0; l <= kMaxLogN1 && e == cudaSuccess; ++l)
        e = cudaFuncSetAttribute(w32::dec_tc32_kernel(l), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(dec_tc32_smem_bytes(kMaxPrimes32)));
    for (int lw = 2; lw <= kMaxL && e == cudaSuccess; lw += 2)
        e = cudaFuncSetAttribute(w32::crt_tc32_kernel(lw), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(w32::crt_tc32_smem_bytes(lw)));
    for (int l = 0; l <= kMaxLogN1 && e == cudaSuccess; ++l)
        e = cudaFuncSetAttribute(w32::batch_dec_tc32_kernel(l), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(dec_tc32_smem_bytes(kMaxPrimes32)));
    for (int n = 1; n <= kBatchRowLogMax && e == cudaSuccess; ++n)
        e = cudaFuncSetAttribute(w32::persistent_rows32_kernel(n), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(w32::row_smem_bytes(kThreads, kBatchRowLogE)));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(w32::k_batch_crt_tc32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(w32::crt_tc32_smem_bytes(30)));
    return e;
}

cudaError_t launch_batch_dec_tc32(const BatchCrtArgs& args, int logN1, int kmax, cudaStream_t s) {
    void* fn = w32::batch_dec_tc32_kernel(logN1);
    if (!fn) return cudaErrorInvalidValue;
    BatchCrtArgs a = args;
    void* params[] = {&a};
    return launch_pdl(fn, args.n_items, kThreads, dec_tc32_smem_bytes(kmax), s, params);
}

cudaError_t launch_persistent_rows32(const BatchArgs& args, int logN2, int ctas, cudaStream_t s) {
    void* fn = w32::persistent_rows32_kernel(logN2);
    if (!fn) return cudaErrorInvalidValue;
    BatchArgs a = args;
    void* params[] = {&a};
    return launch_pdl(fn, ctas, kThreads, w32::row_smem_bytes(kThreads, kBatchRowLogE), s, params);
}

cudaError_t persistent_rows32_occupancy(int logN2, int* ctas_per_sm) {
    void* fn = w32::persistent_rows32_kernel(logN2);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, kThreads,
                                                         w32::row_smem_bytes(kThreads, kBatchRowLogE));
}

cudaError_t launch_batch_crt_tc32(const BatchCrtArgs& args, int lw_max, cudaStream_t s) {
    BatchCrtArgs a = args;
    void* params[] = {&a};
    return launch_pdl(reinterpret_cast<void*>(&w32::k_batch_crt_tc32), args.n_items, kThreads,
                      w32::crt_tc32_smem_bytes(lw_max), s, params);
}

cudaError_t launch_residues32(const ProductDesc& d, const Tables& t, int logN1, cudaStream_t s, int first, int count,
                              int tile0, int tiles) {
    void* fn = w32::dec_tc32_kernel(logN1);
    if (!fn || !t.res_w32 || int(d.k) > kMaxPrimes32) return cudaErrorInvalidValue;
    ProductDesc dd = d;
    Tables tt = t;
    void* args[] = {&dd, &tt, &first, &tile0, &tiles};
    return launch_pdl(fn, count * tiles, kThreads, dec_tc32_smem_bytes(int(d.k)), s, args);
}

cudaError_t launch_row32(const ProductDesc& d, const Tables& t, const RowConfig& cfg, cudaStream_t s) {
    void* fn = row32_kernel(cfg);
    if (!fn) return cudaErrorInvalidValue;
    const Geometry g = geometry(int(d.logN), int(d.k), cfg);
    ProductDesc dd = d;
    Tables tt = t;
    void* args[] = {&dd, &tt};
    return launch_pdl(fn, g.row_ctas, cfg.threads, w32::row_smem_bytes(cfg.threads, cfg.logE), s, args);
}

cudaError_t launch_crt32(const ProductDesc& d, const Tables& t, int tiles, cudaStream_t s) {
    void* fn = w32::crt_tc32_kernel(int(d.LW));
    if (!fn || !d.crt_b || !d.qc32) return cudaErrorInvalidValue;
    ProductDesc dd = d;
    Tables tt = t;
    void* args[] = {&dd, &tt};
    return launch_pdl(fn, tiles, kThreads, w32::crt_tc32_smem_bytes(int(d.LW)), s, args);
}

}  // namespace nc
