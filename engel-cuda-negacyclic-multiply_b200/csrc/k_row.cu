// Stage 2 kernels: k_row<LOG_N2, LOG_E, THREADS> (forward a, forward b, pointwise, inverse).
#include "kernel_registry.h"
#include "stages.cuh"

namespace nc {

// Resident CTAs per SM the register allocation aims at: radix-8 passes in 256-thread CTAs fit three
// (80 registers a thread; k_row<11,3,256> at N = 2^16: 69.6 us against 71.7 us at two), radix-16
// passes keep two (128 registers; at 80 they spill about 500 bytes a thread).
template <int LOG_N2, int LOG_E, int THREADS>
__global__ void __launch_bounds__(THREADS, (THREADS == 256 ? (LOG_E == 3 ? 3 : 2) : 1)) k_row(ProductDesc d, Tables t) {
    extern __shared__ __align__(16) uint8_t smem[];
    pdl_trigger();
    row_blocks<LOG_N2, LOG_E, THREADS>(d, t, int(blockIdx.x), smem);
}

// Radix 16 with 256 threads for every block size, radix 8 with 256 threads for 64..2048-residue
// blocks, and 512-thread variants for the large blocks.
#define NC_ROW_VARIANTS(X)                                                                                     \
    X(1, 4, 256) X(2, 4, 256) X(3, 4, 256) X(4, 4, 256) X(5, 4, 256) X(6, 4, 256) X(7, 4, 256) X(8, 4, 256)  \
    X(9, 4, 256) X(10, 4, 256) X(11, 4, 256) X(12, 4, 256) X(6, 3, 256) X(7, 3, 256) X(8, 3, 256)           \
    X(9, 3, 256) X(10, 3, 256) X(11, 3, 256) X(9, 3, 512) X(10, 3, 512) X(11, 3, 512) X(12, 3, 512)          \
    X(9, 4, 512) X(10, 4, 512) X(11, 4, 512) X(12, 4, 512) X(13, 4, 512)

void* row_kernel(const RowConfig& c) {
#define NC_ROW(n, e, th) \
    if (c.logN2 == n && c.logE == e && c.threads == th) return reinterpret_cast<void*>(&k_row<n, e, th>);
    NC_ROW_VARIANTS(NC_ROW)
#undef NC_ROW
    return nullptr;
}

std::vector<RowConfig> all_row_variants() {
    std::vector<RowConfig> v;
#define NC_ROW_LIST(n, e, th) v.push_back(RowConfig{n, e, th});
    NC_ROW_VARIANTS(NC_ROW_LIST)
#undef NC_ROW_LIST
    return v;
}

cudaError_t prepare_row(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = upload_prime_constants(pc, pow32);
    for (const RowConfig& c : all_row_variants()) {
        if (e != cudaSuccess) break;
        e = cudaFuncSetAttribute(row_kernel(c), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(row_smem_bytes(c.threads, c.logE)));
    }
    return e;
}

}  // namespace nc
