// Stage 3 kernels: k_crt<LW> (inverse column stages + CRT + Barrett), grid = tiles.
#include "kernel_registry.h"
#include "stages.cuh"

namespace nc {

template <int LW>
__global__ void __launch_bounds__(kThreads, 2) k_crt(ProductDesc d, Tables t) {
    extern __shared__ __align__(16) uint8_t smem[];
    pdl_trigger();
    crt_coeffs<LW>(d, t, int(blockIdx.x), smem);
}

void* crt_kernel(int LW) {
    switch (LW) {
#define NC_CRT(n) \
    case n: return reinterpret_cast<void*>(&k_crt<n>);
        NC_LW_CASES(NC_CRT)
#undef NC_CRT
        default: return nullptr;
    }
}

cudaError_t prepare_crt(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = upload_prime_constants(pc, pow32);
    for (int lw = 2; lw <= kMaxL && e == cudaSuccess; lw += 2)
        e = cudaFuncSetAttribute(crt_kernel(lw), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(crt_smem_bytes(kMaxPrimes)));
    return e;
}

}  // namespace nc
