// Batched kernels: the row stage of every product of a batch (and the residue stage of products on
// the integer residue engine) in persistent launches, then the CRT stage of every product in one
// launch per CRT engine. Residues on the tensor cores run before, in k_batch_dec_tc (k_dec_tc.cu);
// products of N >= 2^15 take the plain path's launches instead (batch.cu). When every residue is
// made on the tensor cores, the row items run in one k_persistent_rows<logN2> launch per row-block
// size present (no waits); otherwise k_persistent runs every residue and row item.
//
// k_persistent: the host lays out a work queue of items (stage, product, index): all residue
// items of every product, then all row items. CTAs (as many as fit on the GPU at once) take items
// in queue order with one atomic. A row item of product p may start once every residue item of p
// is done; the CTA's first thread polls p's counter. Every item a CTA waits for was taken earlier
// by a CTA that is running and waits on nothing later in the queue, so the waits always end. A
// wait is still bounded: past kSpinLimit polls (about two seconds) the CTA records an error, skips
// the item, and every later wait returns at once; the host reports the error after the launch.
//
// CRT launches (after the persistent launch on the same stream, so every row item is done): one
// CTA per (product, 256-coefficient tile). Products with a tensor-core table and at most 30 limbs
// run crt_coeffs_tc in k_batch_crt_tc (256 tensor-memory columns per CTA); the others run
// crt_coeffs in k_batch_crt. Keeping the CRT out of the persistent loop keeps its register-heavy
// code out of the residue and row items' register allocation.
#include "crt_tc.cuh"
#include "kernel_registry.h"
#include "stages.cuh"

namespace nc {

constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 only. True once *ctr >= need; false after kSpinLimit polls or once an error is set.
// The first wait to give up records what it waited for: error[1] = stage << 28 | product,
// error[2] = the count it last saw, error[3] = the count it needed.
__device__ bool wait_count(const uint32_t* ctr, uint32_t need, uint32_t* error, uint32_t what) {
    uint32_t seen = 0;
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        seen = ld_acquire(ctr);
        if (seen >= need) return true;
        if (ld_acquire(error) != 0) return false;
        __nanosleep(it < 64 ? 64 : 512);
    }
    if (atomicCAS(error, 0u, 1u) == 0u) {
        error[1] = what;
        error[2] = seen;
        error[3] = need;
    }
    return false;
}

template <int LW>
__device__ __forceinline__ void batch_dec(const BatchProduct& bp, const Tables& t, int idx, uint8_t* smem) {
    const int operand = int(bp.first_operand) + idx / int(bp.tiles);
    dec_tile<LW>(bp.d, t, operand, idx % int(bp.tiles), smem);
}

// A residue item (a product on the integer residue engine) or a row item of any row-block size.
__device__ __forceinline__ void batch_item(uint32_t stage, const BatchProduct& bp, const Tables& t, int idx,
                                           uint8_t* smem) {
    if (stage == kItemDec) {
        switch (bp.d.LW) {
#define NC_B_DEC(n) \
    case n: batch_dec<n>(bp, t, idx, smem); break;
            NC_LW_CASES(NC_B_DEC)
#undef NC_B_DEC
            default: break;
        }
    } else if (stage == kItemRow) {
        switch (bp.d.logN2) {
#define NC_B_ROW(n) \
    case n: row_blocks<n, kBatchRowLogE, kThreads>(bp.d, t, idx, smem); break;
            NC_B_ROW(1) NC_B_ROW(2) NC_B_ROW(3) NC_B_ROW(4) NC_B_ROW(5) NC_B_ROW(6)
            NC_B_ROW(7) NC_B_ROW(8) NC_B_ROW(9) NC_B_ROW(10) NC_B_ROW(11)
#undef NC_B_ROW
            default: break;
        }
    }
}

// Queues with residue items (products on the integer residue engine): residue items, then row
// items of any row-block size. The item's product descriptor is copied into shared memory once per
// item, and the stages read its fields from there.
__global__ void __launch_bounds__(kThreads, 2) k_persistent(BatchArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    pdl_trigger();
    __shared__ int s_item;
    __shared__ int s_go;
    __shared__ __align__(16) BatchProduct s_bp;
    constexpr int kWords = int(sizeof(BatchProduct) / 4);
    static_assert(sizeof(BatchProduct) % 4 == 0, "descriptor copied in words");
    for (;;) {
        if (threadIdx.x == 0) s_item = int(atomicAdd(a.head, 1u));
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const uint2 w = __ldg(a.items + it);
        const uint32_t stage = w.x >> 28;
        const uint32_t prod = w.x & 0x0fffffffu;
        if (threadIdx.x < kWords)
            reinterpret_cast<uint32_t*>(&s_bp)[threadIdx.x] =
                __ldg(reinterpret_cast<const uint32_t*>(a.products + prod) + threadIdx.x);
        if (threadIdx.x == 0) {
            bool ok = true;
            if (stage == kItemRow) ok = wait_count(a.counters + 2 * prod, __ldg(&a.products[prod].n_dec), a.error, w.x);
            s_go = ok ? 1 : 0;
        }
        __syncthreads();
        if (s_go) {
            batch_item(stage, s_bp, a.tables, int(w.y), smem);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0 && stage == kItemDec) atomicAdd(a.counters + 2 * prod, 1u);
        }
        __syncthreads();  // s_item / s_go are rewritten by the next round
    }
}

// Row items alone, every one of them with row blocks of 2^LOG_N2 residues (the batch launches one
// of these per row-block size present, after the residue launches): no item waits, and one
// instantiation per kernel keeps the row stage at 80 registers without spills, three CTAs per SM
// (the switch over every size in k_persistent<false> spills about 1.2 KB a thread).
template <int LOG_N2>
__global__ void __launch_bounds__(kThreads, 3) k_persistent_rows(BatchArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    pdl_trigger();
    __shared__ int s_item;
    __shared__ __align__(16) BatchProduct s_bp;
    constexpr int kWords = int(sizeof(BatchProduct) / 4);
    for (;;) {
        if (threadIdx.x == 0) s_item = int(atomicAdd(a.head, 1u));
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const uint2 w = __ldg(a.items + it);
        if (threadIdx.x < kWords)
            reinterpret_cast<uint32_t*>(&s_bp)[threadIdx.x] =
                __ldg(reinterpret_cast<const uint32_t*>(a.products + (w.x & 0x0fffffffu)) + threadIdx.x);
        __syncthreads();
        row_blocks<LOG_N2, kBatchRowLogE, kThreads>(s_bp.d, a.tables, int(w.y), smem);
        __syncthreads();  // s_item and s_bp are rewritten by the next round
    }
}

static void* persistent_rows_kernel(int logN2) {
    switch (logN2) {
#define NC_P_ROWS(n) \
    case n: return reinterpret_cast<void*>(&k_persistent_rows<n>);
        NC_P_ROWS(1) NC_P_ROWS(2) NC_P_ROWS(3) NC_P_ROWS(4) NC_P_ROWS(5) NC_P_ROWS(6)
        NC_P_ROWS(7) NC_P_ROWS(8) NC_P_ROWS(9) NC_P_ROWS(10) NC_P_ROWS(11)
#undef NC_P_ROWS
        default: return nullptr;
    }
}

__global__ void __launch_bounds__(kThreads, 2) k_batch_crt(BatchCrtArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    pdl_trigger();
    const uint2 w = __ldg(a.items + blockIdx.x);
    const BatchProduct& bp = a.products[w.x];
    switch (bp.d.LW) {
#define NC_B_CRT(n) \
    case n: crt_coeffs<n>(bp.d, a.tables, int(w.y), smem); break;
        NC_LW_CASES(NC_B_CRT)
#undef NC_B_CRT
        default: break;
    }
}

__global__ void __launch_bounds__(kThreads, 2) k_batch_crt_tc(BatchCrtArgs a) {
#if NC_HAS_TCGEN05
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(
                         crt_tc_detail::smem_u32(&taddr_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(crt_tc_detail::smem_u32(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // triggered only once the CTA holds its tensor memory (see k_dec_tc.cu)
    pdl_trigger();
    const uint32_t taddr = taddr_slot;
    const uint2 w = __ldg(a.items + blockIdx.x);
    const BatchProduct& bp = a.products[w.x];
    switch (bp.d.LW) {
#define NC_B_CRT_TC(n)                                                        \
    case n:                                                                   \
        if constexpr (crt_tc_tmem_cols(n) == 256)                             \
            crt_coeffs_tc<n>(bp.d, a.tables, int(w.y), smem, taddr, &bar, 0); \
        break;
        NC_LW_CASES(NC_B_CRT_TC)
#undef NC_B_CRT_TC
        default: break;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(taddr) : "memory");
#endif
}

cudaError_t launch_batch_crt(const BatchCrtArgs& args, bool tensor_cores, size_t smem, cudaStream_t s) {
    BatchCrtArgs a = args;
    void* params[] = {&a};
    void* fn = tensor_cores ? reinterpret_cast<void*>(&k_batch_crt_tc) : reinterpret_cast<void*>(&k_batch_crt);
    return launch_pdl(fn, args.n_items, kThreads, smem, s, params);
}

cudaError_t prepare_persistent(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = upload_prime_constants(pc, pow32);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smax(dec_smem_bytes(kMaxPrimes), row_smem_bytes(kThreads, kBatchRowLogE))));
    for (int n = 1; n <= kBatchRowLogMax && e == cudaSuccess; ++n)
        e = cudaFuncSetAttribute(persistent_rows_kernel(n), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(row_smem_bytes(kThreads, kBatchRowLogE)));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_crt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(crt_smem_bytes(kMaxPrimes)));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_crt_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(crt_tc_smem_bytes(30)));
    return e;
}

// Launch with `ctas` persistent CTAs and `smem` dynamic shared memory; `with_dec` when the queue
// holds residue items.
cudaError_t launch_persistent(const BatchArgs& args, int ctas, size_t smem, cudaStream_t s) {
    BatchArgs a = args;
    void* params[] = {&a};
    return launch_pdl(reinterpret_cast<void*>(&k_persistent), ctas, kThreads, smem, s, params);
}

cudaError_t launch_persistent_rows(const BatchArgs& args, int logN2, int ctas, cudaStream_t s) {
    BatchArgs a = args;
    void* params[] = {&a};
    void* fn = persistent_rows_kernel(logN2);
    if (!fn) return cudaErrorInvalidValue;
    return launch_pdl(fn, ctas, kThreads, row_smem_bytes(kThreads, kBatchRowLogE), s, params);
}

cudaError_t persistent_rows_occupancy(int logN2, int* ctas_per_sm) {
    void* fn = persistent_rows_kernel(logN2);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, kThreads, row_smem_bytes(kThreads, kBatchRowLogE));
}

cudaError_t persistent_occupancy(size_t smem, int* ctas_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, k_persistent, kThreads, smem);
}

}  // namespace nc
