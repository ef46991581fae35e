// Stage 3 on the tensor cores (inverse column stages + CRT + Barrett) as a CTA-level device
// function, one thread per coefficient of a 256-coefficient tile; k_crt_tc (plain path) and the
// batched CRT launch call it.
//
// The CRT accumulation acc = sum_i v_i (M/p_i mod q) (solve.cu:752-836 forms the same sum with
// 34-limb multiply-adds) is an exact u8 x u8 contraction. With v_i = sum_a v_{i,a} 2^(8a) (8
// bytes) and M_i = (M/p_i) mod q = sum_b m_{i,b} 2^(8b) (4 L bytes),
//
//   acc = sum_c 2^(8c) S_c,   S_c = sum_i sum_{a + b = c} v_{i,a} m_{i,b},
//
// i.e. S = A B with A[n][8i + a] = v_{i,a} of coefficient n (K = 8k <= 256 bytes) and the per-plan
// table B[c][8i + a] = m_{i, c - a} (NC = 4 LW + 7 rounded up to 16 output columns). Every
// S_c < 8 k 255^2 < 2^24, so s32 accumulation is exact and the folded sum is the same integer the
// integer-pipe kernel forms. The tile's 256 coefficients are two M = 128 MMAs per 32-byte K slice
// (tcgen05.mma.cta_group::1.kind::i8), accumulators in tensor memory; each thread then folds its
// row of S into 32-bit words with one carry pass, adds K (-M mod q) and runs the Barrett reduction
// of crt_coeffs. If the bounded wait for the MMAs gives up, the thread forms the sum with the
// integer carry chains instead, so the result never depends on the wait.
#pragma once

#include "stages.cuh"

namespace nc {

namespace crt_tc_detail {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// K-major operand without swizzling: 8-row x 16-byte core matrices, `lbo` bytes between the two K
// chunks of one MMA, `sbo` bytes between 8-row groups, descriptor version 1, layout type 0.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

constexpr uint32_t kMmaWaitLimit = 1u << 22;

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ bool mma_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kMmaWaitLimit; ++it) {
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

// Byte offset of (row, byte) in an A half-tile: [16 row groups][16 K chunks][8 rows][16 B].
__device__ __forceinline__ int a_offset(int row, int byte) {
    return (row >> 3) * 2048 + (byte >> 4) * 128 + (row & 7) * 16 + (byte & 15);
}

// Inverse column stages of items (prime i, column j), then v_i = r_i y_i mod p_i of each of the
// column's N1 coefficients, stored as 8 bytes at K offset 8 i of the coefficient's row of A.
template <int LOG_N1>
__device__ void crt_columns_tc(const ProductDesc& d, const Tables& t, int j0, int T, const uint64_t* s_y,
                               const uint64_t* s_ys, const uint64_t* s_p, uint8_t* sA) {
    constexpr int N1 = 1 << LOG_N1;
    const int N = 1 << d.logN;
    const int N2 = N >> LOG_N1;
    const int C = T >> LOG_N1;
    const int k = int(d.k);
    if constexpr (LOG_N1 == 5) {
        // 32-point columns on two adjacent lanes: lane h loads rows [16h, 16h + 16) and runs the
        // inverse stages of its half-subtree (twiddle root 2 + h); then the last stage's pairs
        // (u, u + 16) are split between the lanes (lane 0: u < 8, lane 1: 8 <= u < 16) with one
        // exchange of eight values. Pairs never straddle a warp (2 k C is even).
        const int total = 2 * k * C;
        const int lane = int(threadIdx.x) & 31;
        for (int w0 = int(threadIdx.x) & ~31; w0 < total; w0 += int(blockDim.x)) {
            const int w = w0 + lane;
            const bool active = w < total;
            const int item = active ? w >> 1 : 0, h = w & 1;
            const int i = item / C, j = item - i * C;
            const uint64_t* row = d.ra + size_t(i) * N + j0 + j + size_t(16 * h) * N2;
            uint64_t v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = active ? __ldcg(row + size_t(u) * N2) : 0;
            const uint64_t p = s_p[i], p2 = 2 * p;
            const ulonglong2* tw = t.inv + size_t(i) * kMaxN;
            column_inverse_root<4>(tw, 2 + h, p, v);
            const ulonglong2 w1 = __ldg(tw + 1);
            const uint64_t y = s_y[i], ys = s_ys[i];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint64_t got = shfl_pair(h ? v[e] : v[8 + e]);
                uint64_t lo = h ? got : v[e], hi = h ? v[8 + e] : got;  // rows 8h + e and 8h + e + 16
                gs_bfly(lo, hi, w1.x, w1.y, p, p2);
                if (active) {
                    const int tl = (8 * h + e) * C + j, th = (8 * h + e + 16) * C + j;
                    *reinterpret_cast<uint64_t*>(sA + (tl >> 7) * kCrtTcHalfBytes + a_offset(tl & 127, 8 * i)) =
                        csub(shoup_lazy(lo, y, ys, p), p);
                    *reinterpret_cast<uint64_t*>(sA + (th >> 7) * kCrtTcHalfBytes + a_offset(th & 127, 8 * i)) =
                        csub(shoup_lazy(hi, y, ys, p), p);
                }
            }
        }
        return;
    }
    for (int w = threadIdx.x; w < k * C; w += blockDim.x) {
        const int i = w / C, j = w - i * C;
        const uint64_t* row = d.ra + size_t(i) * N + j0 + j;
        uint64_t v[N1];
#pragma unroll
        for (int u = 0; u < N1; ++u) v[u] = __ldcg(row + size_t(u) * N2);
        const uint64_t p = s_p[i];
        if (LOG_N1 > 0) column_inverse<LOG_N1>(t.inv + size_t(i) * kMaxN, p, v);
        const uint64_t y = s_y[i], ys = s_ys[i];
#pragma unroll
        for (int u = 0; u < N1; ++u) {
            const int tc = u * C + j;
            const uint64_t vi = csub(shoup_lazy(v[u], y, ys, p), p);
            *reinterpret_cast<uint64_t*>(sA + (tc >> 7) * kCrtTcHalfBytes + a_offset(tc & 127, 8 * i)) = vi;
        }
    }
}

}  // namespace crt_tc_detail

// One 256-coefficient tile (index `tile`) with every thread of a 256-thread CTA. The caller owns
// crt_tc_tmem_cols(LW) columns of tensor memory at `taddr` and an initialised mbarrier `bar`
// whose phase `parity` the MMAs of this call complete.
template <int LW>
__device__ void crt_coeffs_tc(const ProductDesc& d, const Tables& t, int tile, uint8_t* smem, uint32_t taddr,
                              uint64_t* bar, uint32_t parity) {
    constexpr int W = LW + kAccExtra;
    constexpr int NC = crt_tc_cols(LW);
    constexpr uint32_t kHalfCol = crt_tc_tmem_cols(LW) / 2;  // second accumulator's first column
    const int N = 1 << d.logN;
    const int logN1 = int(d.logN) - int(d.logN2);
    const int N2 = N >> logN1;
    const int T = N < kTile ? N : kTile;
    const int C = T >> logN1;
    const int k = int(d.k), L = int(d.L);
    const int j0 = tile * C;

    uint8_t* sA = smem;                                    // two half-tiles of 128 rows x 256 K bytes
    uint8_t* sB = smem + 2 * kCrtTcHalfBytes;              // NC / 8 column groups x 2048 bytes
    uint64_t* s_y = reinterpret_cast<uint64_t*>(sB + NC * 256);
    uint64_t* s_ys = s_y + kCrtTcMaxPrimes;
    uint64_t* s_p = s_ys + kCrtTcMaxPrimes;
    uint32_t* s_negm = reinterpret_cast<uint32_t*>(s_p + kCrtTcMaxPrimes);
    uint32_t* s_q = s_negm + kMqStride;
    uint32_t* s_mu = s_q + kMqStride;
    const int tid = int(threadIdx.x), warp = tid >> 5;

    __syncthreads();  // shared memory of a previous item is free
    const QConst* qc = d.qc;
    for (int w = tid; w < k; w += blockDim.x) {
        s_y[w] = __ldg(qc->y + w);
        s_ys[w] = __ldg(qc->ys + w);
        s_p[w] = __ldg(t.primes + w);
    }
    for (int w = tid; w < kMqStride; w += blockDim.x) {
        s_negm[w] = __ldg(qc->neg_m + w);
        s_q[w] = __ldg(qc->q + w);
    }
    if (tid < 4) s_mu[tid] = __ldg(qc->mu + tid);
    // the table is first read by the MMAs: its copy runs behind the column stages
    for (int w = tid; w < NC * 16; w += blockDim.x) crt_tc_detail::cp_async16(sB + 16 * w, d.crt_b + w);
    asm volatile("cp.async.commit_group;" ::: "memory");
    __syncthreads();
    pdl_wait();  // the residues come from the stream's previous kernel

    switch (logN1) {
        case 0: crt_tc_detail::crt_columns_tc<0>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 1: crt_tc_detail::crt_columns_tc<1>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 2: crt_tc_detail::crt_columns_tc<2>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 3: crt_tc_detail::crt_columns_tc<3>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        case 4: crt_tc_detail::crt_columns_tc<4>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
        default: crt_tc_detail::crt_columns_tc<5>(d, t, j0, T, s_y, s_ys, s_p, sA); break;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A's and B's writes -> MMA reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (tid == 0) {
        // kind::i8: D s32 (bits 4-5 = 2), A and B u8, K-major; N >> 3 at bit 17, M >> 4 at bit 24
        const uint32_t idesc = (2u << 4) | (uint32_t(NC >> 3) << 17) | (uint32_t(128 >> 4) << 24);
        const int slices = (8 * k + 31) / 32;
        const uint32_t b0 = crt_tc_detail::smem_u32(sB);
        for (int h = 0; h < (T > 128 ? 2 : 1); ++h) {
            const uint32_t a0 = crt_tc_detail::smem_u32(sA + h * kCrtTcHalfBytes);
            for (int s = 0; s < slices; ++s) {
                const uint64_t da = crt_tc_detail::kmajor_desc(a0 + uint32_t(s) * 256u, 128u, 2048u);
                const uint64_t db = crt_tc_detail::kmajor_desc(b0 + uint32_t(s) * 256u, 128u, 2048u);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr + uint32_t(h) * kHalfCol),
                    "l"(da), "l"(db), "r"(idesc), "r"(s));
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         crt_tc_detail::smem_u32(bar))
                     : "memory");
    }

    // While the MMAs run: this thread's coefficient, its v_i, and the CRT quotient estimate.
    const int tc = tid;
    const int half = tc >> 7;
    const uint8_t* arow = sA + half * kCrtTcHalfBytes + crt_tc_detail::a_offset(tc & 127, 0);
    uint64_t frac = 0;
#pragma unroll 1
    for (int i = 0; i < k; ++i) {
        const uint64_t v = *reinterpret_cast<const uint64_t*>(arow + (i >> 1) * 128 + (i & 1) * 8);
        frac += (uint64_t(uint32_t(v >> 30)) * c_pc[i].g) >> 31;  // 2^32 v / p_i
    }
    const uint32_t kq = uint32_t((frac + (1ull << 31)) >> 32);

    const bool ok = crt_tc_detail::mma_wait(crt_tc_detail::smem_u32(bar), parity);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    uint32_t acc[W];
#pragma unroll
    for (int w = 0; w < W; ++w) acc[w] = 0;
    if (__all_sync(0xffffffffu, ok)) {
        // fold S_c 2^(8c) into 32-bit words: two words per group of eight columns, one carry pass
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
            const uint64_t v = *reinterpret_cast<const uint64_t*>(arow + (i >> 1) * 128 + (i & 1) * 8);
            const uint32_t* M = qc->mq + i * kMqStride;
            uint32_t m[LW];
#pragma unroll
            for (int l = 0; l < LW; ++l) m[l] = __ldg(M + l);
            mac_lo<LW, 0, W>(acc, m, uint32_t(v));
            mac_hi<LW, 1, W>(acc_hi, m, uint32_t(v));
            mac_lo<LW, 1, W>(acc, m, uint32_t(v >> 32));
            mac_hi<LW, 2, W>(acc_hi, m, uint32_t(v >> 32));
        }
        asm volatile("add.cc.u32 %0, %0, %1;" : "+r"(acc[0]) : "r"(acc_hi[0]));
#pragma unroll
        for (int w = 1; w < W - 1; ++w) asm volatile("addc.cc.u32 %0, %0, %1;" : "+r"(acc[w]) : "r"(acc_hi[w]));
        asm volatile("addc.u32 %0, %0, %1;" : "+r"(acc[W - 1]) : "r"(acc_hi[W - 1]));
    }
    // acc += round(sum v_i / p_i) * ((-M) mod q)
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

    // every thread is past its reads of A and of tensor memory: stage the tile's output in A
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

}  // namespace nc
