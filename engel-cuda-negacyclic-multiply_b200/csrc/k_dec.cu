// Stage 1 kernels: k_dec<LW> (residues + forward column stages), grid = operands x tiles.
#include "kernel_registry.h"
#include "stages.cuh"

namespace nc {

// Three CTAs per SM (at most 85 registers a thread; 67 KB of shared memory each at 29 primes):
// the residue loop is latency bound, and the third CTA's warps hide more of it than the
// registers it costs (measured at N = 65536, 868-bit q: 78.1 -> 75.1 us).
template <int LW>
__global__ void __launch_bounds__(kThreads, 3) k_dec(ProductDesc d, Tables t, int first_operand, int tile0, int tiles) {
    extern __shared__ __align__(16) uint8_t smem[];
    pdl_trigger();
    const int operand = first_operand + int(blockIdx.x) / tiles;
    const int tile = tile0 + int(blockIdx.x) % tiles;
    dec_tile<LW>(d, t, operand, tile, smem);
}

void* dec_kernel(int LW) {
    switch (LW) {
#define NC_DEC(n) \
    case n: return reinterpret_cast<void*>(&k_dec<n>);
        NC_LW_CASES(NC_DEC)
#undef NC_DEC
        default: return nullptr;
    }
}

cudaError_t prepare_dec(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = upload_prime_constants(pc, pow32);
    for (int lw = 2; lw <= kMaxL && e == cudaSuccess; lw += 2)
        e = cudaFuncSetAttribute(dec_kernel(lw), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(dec_smem_bytes(kMaxPrimes)));
    return e;
}

}  // namespace nc
