// Stage 3 kernels on the tensor cores: k_crt_tc<LW>, grid = 256-coefficient tiles (see crt_tc.cuh).
#include "crt_tc.cuh"
#include "kernel_registry.h"

namespace nc {

template <int LW>
__global__ void __launch_bounds__(kThreads, 2) k_crt_tc(ProductDesc d, Tables t) {
#if NC_HAS_TCGEN05
    constexpr uint32_t kCols = crt_tc_tmem_cols(LW);
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t taddr_slot;
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         crt_tc_detail::smem_u32(&taddr_slot)),
                     "r"(kCols)
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
    crt_coeffs_tc<LW>(d, t, int(blockIdx.x), smem, taddr, &bar, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kCols) : "memory");
#endif
}

void* crt_tc_kernel(int LW) {
    switch (LW) {
#define NC_CRT_TC(n) \
    case n: return reinterpret_cast<void*>(&k_crt_tc<n>);
        NC_LW_CASES(NC_CRT_TC)
#undef NC_CRT_TC
        default: return nullptr;
    }
}

cudaError_t prepare_crt_tc(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = upload_prime_constants(pc, pow32);
    for (int lw = 2; lw <= kMaxL && e == cudaSuccess; lw += 2)
        e = cudaFuncSetAttribute(crt_tc_kernel(lw), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(crt_tc_smem_bytes(lw)));
    return e;
}

}  // namespace nc
