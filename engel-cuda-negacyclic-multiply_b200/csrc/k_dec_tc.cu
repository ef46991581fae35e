// Stage 1 on the tensor cores: the residues of an operand tile by an exact INT8 contraction, then
// the forward column stages (the same output as k_dec); k_dec_tc<LOG_N1> runs one product (plain
// path), k_batch_dec_tc<LOG_N1> the residue items of a batch.
//
// The residue x_n mod p_i of a coefficient given as 4 L bytes x_{n,b} (little-endian limbs, the
// counterpart of to_residues_tiled_kernel, solve.cu:533-570) is
//
//   x_n = sum_c 2^(8 c) S[n][i,c]  (mod p_i),   S[n][i,c] = sum_b x_{n,b} w_{i,b,c},
//
// with w_{i,b,c} byte c of 2^(8 b) mod p_i. S is a u8 x u8 matrix product: 128 coefficients (M)
// x 128 K bytes (4 L, zero padded) x 8 columns per prime, every S < 128 * 255^2 < 2^23, so the s32
// accumulation in tensor memory is exact. The primes (any count up to 48) go through
// tcgen05.mma kind::i8 in passes of 16 (128 accumulator columns); after each pass the eight warps
// read the partial sums back
// (tcgen05.ld) and fold sum_c 2^(8 c) S_c (< 2^80) into [0, 2p) modulo p_i. The tile is
// C = 128 / N1 columns of all N1 rows of the polynomial (row length N2 = N / N1), as in k_dec, so
// the forward column stages and the residue-row stores follow unchanged.
//
// Operand and weight bytes reach shared memory by cp.async (no register staging). Each prime's
// residues overwrite its own 1 KB of weights once its pass's MMAs have completed. If the bounded
// wait for a pass gives up, each warp forms its
// residues with the integer carry chains of k_dec instead, so the result never depends on it.
#include "batch_types.h"
#include "crt_tc.cuh"
#include "kernel_registry.h"

namespace nc {

namespace {

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

// sum_c 2^(8 c) s[c] mod p = 2^62 - m, for s[c] < 2^23, into [0, 2p). With A = sum_{c<4} and
// B = sum_{c>=4} 2^(8 (c - 4)) s[c] (both < 2^48) the value is A + B 2^32, and since
// 2^62 = m (mod p), B 2^32 = (B >> 30) m + (B mod 2^30) 2^32, so the sum
// A + (B mod 2^30) 2^32 + (B >> 30) m < 2^62 + 2^49 is below 2p: six wide multiply-adds, a
// shift, a mask, one add and one more multiply-add.
__device__ __forceinline__ uint64_t mad_wide(uint32_t a, uint32_t b, uint64_t c) {
    uint64_t d;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t fold_planes(const uint32_t* s, uint32_t m) {
    const uint64_t a = mad_wide(s[3], 1u << 24, mad_wide(s[2], 1u << 16, mad_wide(s[1], 1u << 8, uint64_t(s[0]))));
    const uint64_t b = mad_wide(s[7], 1u << 24, mad_wide(s[6], 1u << 16, mad_wide(s[5], 1u << 8, uint64_t(s[4]))));
    const uint32_t bq = uint32_t(b >> 30);                                      // < 2^18
    const uint64_t r = a + (uint64_t(uint32_t(b) & ((1u << 30) - 1)) << 32);   // < 2^62 + 2^48
    return mad_wide(bq, m, r);
}

// Residue row of prime i in shared memory (128 values), over the prime's own weights.
__device__ __forceinline__ uint64_t* res_row(uint8_t* sB, int i) { return reinterpret_cast<uint64_t*>(sB + i * 1024); }

// Slot of tile row x in prime i's residue row: rows XORed with (i C) mod 16, so that the 32 / C
// primes one warp reads in the column stages (C consecutive rows each) fall on different banks.
__device__ __forceinline__ int res_slot(int i, int x, int C) { return x ^ ((i * C) & 15); }

// One CTA's tile: operand `operand` of product d, 128-coefficient tile `tile`; `bar` and
// `taddr_slot` are the CTA's mbarrier and tensor-memory address slot in shared memory.
template <int LOG_N1>
__device__ __forceinline__ void dec_tc_item(const ProductDesc& d, const Tables& t, int operand, int tile, uint8_t* smem,
                                            uint64_t& bar, uint32_t& taddr_slot) {
    constexpr int N1 = 1 << LOG_N1;
    const int N = 1 << d.logN;
    const int N2 = N >> LOG_N1;
    const int T = N < kDecTcRows ? N : kDecTcRows;
    const int logC = (N < kDecTcRows ? int(d.logN) : 7) - LOG_N1;
    const int C = 1 << logC;
    const int j0 = tile * C;
    const int L = int(d.L), k = int(d.k);
    const int groups = (k + 1) & ~1;
    const uint32_t* x = factor_limbs(d, operand);
    uint64_t* R = factor_residues(d, operand);
    uint8_t* sA = smem;                         // [16 row groups][8 K chunks][8 rows][16 B]
    uint8_t* sB = smem + kDecTcRows * 128;      // [prime][8 K chunks][8 byte planes][16 B]
    uint64_t* s_p = reinterpret_cast<uint64_t*>(sB + groups * 1024);
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
    // The next kernel on the stream may be scheduled only once every CTA of this one holds its
    // tensor memory: a dependent that allocates before its griddepcontrol.wait could otherwise
    // take the columns a CTA of this kernel still waits for, and each would wait on the other.
    __syncthreads();
    pdl_trigger();

    // B: the weight bytes of the first `groups` primes, already in shared-memory order
    for (int q = tid; q < groups * 64; q += kThreads) cp_async16(sB + q * 16, t.res_w + q);
    for (int w = tid; w < k; w += kThreads) s_p[w] = __ldg(t.primes + w);
    pdl_wait();  // the operand and the residue rows belong to the stream's previous kernels
    // A: 16-byte chunk q = (row group, K chunk, row), row m = u C + j is coefficient u N2 + j0 + j
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
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy writes -> MMA reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = taddr_slot;
    const int slices = (kbytes + 31) / 32;

    // passes of 16 primes; warp w reads tensor-memory lanes 32 (w % 4) .. (its coefficient rows)
    // and half w / 4 of the pass's primes
    const int m = 32 * (warp & 3) + lane;
    const int half = warp >> 2;
    bool failed = false;
    for (int g = 0; g * kDecTcPassPrimes < k; ++g) {
        const int i0 = g * kDecTcPassPrimes;
        const int np = k - i0 < kDecTcPassPrimes ? k - i0 : kDecTcPassPrimes;
        if (tid == 0 && !failed) {
            // kind::i8: D s32 (bits 4-5 = 2), A and B u8, K-major; N >> 3 at bit 17, M >> 4 at bit 24
            const uint32_t ng = uint32_t((np + 1) & ~1);
            const uint32_t idesc = (2u << 4) | (ng << 17) | (uint32_t(kDecTcRows >> 4) << 24);
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB + i0 * 1024);
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
        const int ib = i0 + 8 * half;
        const int ie = i0 + np < ib + 8 ? i0 + np : ib + 8;
        if (__all_sync(0xffffffffu, ok)) {
            const uint32_t lane_base = taddr + (uint32_t(32 * (warp & 3)) << 16);
            for (int i = ib; i < ie; i += 2) {
                uint32_t s[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]),
                      "=r"(s[8]), "=r"(s[9]), "=r"(s[10]), "=r"(s[11]), "=r"(s[12]), "=r"(s[13]), "=r"(s[14]),
                      "=r"(s[15])
                    : "r"(lane_base + uint32_t(8 * (i - i0))));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                res_row(sB, i)[res_slot(i, m, C)] = fold_planes(s, uint32_t((uint64_t(1) << 62) - s_p[i]));
                if (i + 1 < ie)
                    res_row(sB, i + 1)[res_slot(i + 1, m, C)] =
                        fold_planes(s + 8, uint32_t((uint64_t(1) << 62) - s_p[i + 1]));
            }
        } else if (m < T) {
            // the wait gave up: this warp's residues by the integer carry chains
            const int n = (m >> logC) * N2 + j0 + (m & (C - 1));
            const uint32_t* row = x + size_t(n) * size_t(L);
            for (int i = ib; i < ie; ++i) {
                uint32_t a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
                for (int l = 0; l < L; ++l) {
                    const uint64_t c = __ldg(t.pow32 + size_t(i) * kMaxL + l);
                    mac_u32x64(__ldg(row + l), uint32_t(c), uint32_t(c >> 32), a0, a1, a2, b0, b1, b2);
                }
                res_row(sB, i)[res_slot(i, m, C)] =
                    reduce_limb_sum(a0, a1, a2, b0, b1, b2, (uint64_t(1) << 62) - s_p[i]);
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
        // 32-point columns on two adjacent lanes (16 values each, like the 16-point case): lane h
        // runs the first stage's butterflies (u, u + 16) for u in [8h, 8h + 8), the lanes swap
        // halves so that lane h holds rows [16h, 16h + 16), and each runs the four remaining stages
        // on its half-subtree (twiddle root 2 + h). Pairs never straddle a warp (2 k C is even).
        const int total = 2 * k * C;
        for (int w0 = tid & ~31; w0 < total; w0 += kThreads) {
            const int w = w0 + lane;
            const bool active = w < total;
            const int item = active ? w >> 1 : 0, h = w & 1;
            const int i = item >> logC, j = item & (C - 1);
            const uint64_t* sr = res_row(sB, i);
            const uint64_t p = s_p[i], p2 = 2 * p;
            const ulonglong2* tw = t.fwd + size_t(i) * kMaxN;
            uint64_t x[8], y[8];
            const ulonglong2 w1 = __ldg(tw + 1);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int u = 8 * h + e;
                x[e] = sr[res_slot(i, u * C + j, C)];
                y[e] = sr[res_slot(i, (u + 16) * C + j, C)];
                ct_bfly(x[e], y[e], w1.x, w1.y, p, p2);
            }
            // lane 0 keeps x (rows 0..7) and takes lane 1's x (8..15); lane 1 takes lane 0's y
            // (16..23) and keeps y (24..31)
            uint64_t v[16];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint64_t send = h ? x[e] : y[e];
                const uint64_t got = (uint64_t(__shfl_xor_sync(0xffffffffu, uint32_t(send >> 32), 1)) << 32) |
                                     __shfl_xor_sync(0xffffffffu, uint32_t(send), 1);
                v[e] = h ? got : x[e];
                v[8 + e] = h ? y[e] : got;
            }
            column_forward_root<4>(tw, 2 + h, p, v);
            if (active) {
                uint64_t* out = R + size_t(i) * N + j0 + j + size_t(16 * h) * N2;
#pragma unroll
                for (int u = 0; u < 16; ++u) __stcg(out + size_t(u) * N2, v[u]);
            }
        }
    } else {
        for (int w = tid; w < k * C; w += kThreads) {
            const int i = w >> logC, j = w & (C - 1);
            const uint64_t* sr = res_row(sB, i);
            uint64_t v[N1];
#pragma unroll
            for (int u = 0; u < N1; ++u) v[u] = sr[res_slot(i, u * C + j, C)];
            if (LOG_N1 > 0) column_forward<LOG_N1>(t.fwd + size_t(i) * kMaxN, s_p[i], v);
            uint64_t* out = R + size_t(i) * N + j0 + j;
#pragma unroll
            for (int u = 0; u < N1; ++u) __stcg(out + size_t(u) * N2, v[u]);
        }
    }
}

// Four CTAs per SM (64 registers; tensor memory holds four). The 32-point columns (two lanes of
// 16 values each) spill about 130 bytes a thread there, and still run faster than at three CTAs
// (80 registers, no spills): N = 2^16, both operands, 47.1 -> 45.1 us.
#define NC_DEC_TC_BOUNDS(LOG_N1) __launch_bounds__(kThreads, 4)

// Plain path: one product, grid = operands x tiles, tiles tile0 .. tile0 + tiles - 1 of each operand.
template <int LOG_N1>
__global__ void NC_DEC_TC_BOUNDS(LOG_N1) k_dec_tc(ProductDesc d, Tables t, int first_operand, int tile0, int tiles) {
#if NC_HAS_TCGEN05
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    dec_tc_item<LOG_N1>(d, t, first_operand + int(blockIdx.x) / tiles, tile0 + int(blockIdx.x) % tiles, smem, bar,
                        taddr_slot);
#endif
}

// Batches: one CTA per item (x = product, y = operand * tiles + tile), every product of the launch
// with the same column length N1.
template <int LOG_N1>
__global__ void NC_DEC_TC_BOUNDS(LOG_N1) k_batch_dec_tc(BatchCrtArgs a) {
#if NC_HAS_TCGEN05
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    const uint2 w = __ldg(a.items + blockIdx.x);
    const BatchProduct& bp = a.products[w.x];
    const int tiles = int(bp.tiles_tc);
    dec_tc_item<LOG_N1>(bp.d, a.tables, int(bp.first_operand) + int(w.y) / tiles, int(w.y) % tiles, smem, bar,
                        taddr_slot);
#endif
}

void* batch_dec_tc_kernel(int logN1) {
    switch (logN1) {
        case 0: return reinterpret_cast<void*>(&k_batch_dec_tc<0>);
        case 1: return reinterpret_cast<void*>(&k_batch_dec_tc<1>);
        case 2: return reinterpret_cast<void*>(&k_batch_dec_tc<2>);
        case 3: return reinterpret_cast<void*>(&k_batch_dec_tc<3>);
        case 4: return reinterpret_cast<void*>(&k_batch_dec_tc<4>);
        case 5: return reinterpret_cast<void*>(&k_batch_dec_tc<5>);
        default: return nullptr;
    }
}

}  // namespace

void* dec_tc_kernel(int logN1) {
    switch (logN1) {
        case 0: return reinterpret_cast<void*>(&k_dec_tc<0>);
        case 1: return reinterpret_cast<void*>(&k_dec_tc<1>);
        case 2: return reinterpret_cast<void*>(&k_dec_tc<2>);
        case 3: return reinterpret_cast<void*>(&k_dec_tc<3>);
        case 4: return reinterpret_cast<void*>(&k_dec_tc<4>);
        case 5: return reinterpret_cast<void*>(&k_dec_tc<5>);
        default: return nullptr;
    }
}

cudaError_t prepare_dec_tc(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = upload_prime_constants(pc, pow32);
    for (int l = 0; l <= kMaxLogN1 && e == cudaSuccess; ++l) {
        e = cudaFuncSetAttribute(dec_tc_kernel(l), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(dec_tc_smem_bytes(kMaxPrimes)));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(batch_dec_tc_kernel(l), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(dec_tc_smem_bytes(kMaxPrimes)));
    }
    return e;
}

cudaError_t launch_batch_dec_tc(const BatchCrtArgs& args, int logN1, size_t smem, cudaStream_t s) {
    void* fn = batch_dec_tc_kernel(logN1);
    if (!fn) return cudaErrorInvalidValue;
    if (args.n_items <= 0) return cudaSuccess;
    BatchCrtArgs a = args;
    void* params[] = {&a};
    return launch_pdl(fn, args.n_items, kThreads, smem, s, params);
}

}  // namespace nc
