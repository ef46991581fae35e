// Plain per-call kernels: one launch per stage, grid = the stage's work items.
#include <cuda_runtime.h>

#include "kernels.h"
#include "stages.cuh"

namespace nc {

template <int LOG_N1>
__global__ void __launch_bounds__(kThreads, 2) k_dec(ProductDesc d, Tables t, int first_operand, int tiles) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int operand = first_operand + int(blockIdx.x) / tiles;
    const int tile = int(blockIdx.x) % tiles;
    dec_tile<LOG_N1>(d, t, operand, tile, smem);
}

template <int LOG_N2>
__global__ void __launch_bounds__(kThreads, 2) k_row(ProductDesc d, Tables t) {
    extern __shared__ __align__(16) uint8_t smem[];
    row_blocks<LOG_N2>(d, t, int(blockIdx.x), smem);
}

template <int LW>
__global__ void __launch_bounds__(kThreads, 2) k_crt(ProductDesc d, Tables t) {
    extern __shared__ __align__(16) uint8_t smem[];
    crt_coeffs<LW>(d, t, int(blockIdx.x), smem);
}

namespace {

template <int LOG_N1>
void* dec_fn() {
    return reinterpret_cast<void*>(&k_dec<LOG_N1>);
}

void* dec_kernel(int logN1) {
    switch (logN1) {
        case 0: return dec_fn<0>();
        case 1: return dec_fn<1>();
        case 2: return dec_fn<2>();
        case 3: return dec_fn<3>();
        default: return dec_fn<4>();
    }
}

void* row_kernel(int logN2) {
    switch (logN2) {
#define NC_ROW(n) \
    case n: return reinterpret_cast<void*>(&k_row<n>);
        NC_ROW(1) NC_ROW(2) NC_ROW(3) NC_ROW(4) NC_ROW(5) NC_ROW(6)
        NC_ROW(7) NC_ROW(8) NC_ROW(9) NC_ROW(10) NC_ROW(11) NC_ROW(12)
#undef NC_ROW
        default: return nullptr;
    }
}

void* crt_kernel(int LW) {
    switch (LW) {
#define NC_CRT(n) \
    case n: return reinterpret_cast<void*>(&k_crt<n>);
        NC_CRT(2) NC_CRT(4) NC_CRT(6) NC_CRT(8) NC_CRT(10) NC_CRT(12) NC_CRT(14) NC_CRT(16)
        NC_CRT(18) NC_CRT(20) NC_CRT(22) NC_CRT(24) NC_CRT(26) NC_CRT(28) NC_CRT(30) NC_CRT(32)
#undef NC_CRT
        default: return nullptr;
    }
}

cudaError_t launch(void* fn, int grid, size_t smem, cudaStream_t s, void** args) {
    if (grid <= 0) return cudaSuccess;
    return cudaLaunchKernel(fn, dim3(unsigned(grid)), dim3(kThreads), args, smem, s);
}

}  // namespace

cudaError_t prepare_plain_kernels() {
    cudaError_t e = cudaSuccess;
    for (int n = 0; n <= 4 && e == cudaSuccess; ++n)
        e = cudaFuncSetAttribute(dec_kernel(n), cudaFuncAttributeMaxDynamicSharedMemorySize, int(dec_smem_bytes()));
    for (int n = 1; n <= kRowLogMax && e == cudaSuccess; ++n)
        e = cudaFuncSetAttribute(row_kernel(n), cudaFuncAttributeMaxDynamicSharedMemorySize, int(row_smem_bytes()));
    for (int lw = 2; lw <= kMaxL && e == cudaSuccess; lw += 2)
        e = cudaFuncSetAttribute(crt_kernel(lw), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(crt_smem_bytes(kMaxPrimes)));
    return e;
}

cudaError_t launch_product(const ProductDesc& d, const Tables& t, cudaStream_t s, cudaEvent_t* ev) {
    const Geometry g = geometry(int(d.logN), int(d.k));
    ProductDesc dd = d;
    Tables tt = t;
    cudaError_t e;
    if (ev && (e = cudaEventRecord(ev[0], s)) != cudaSuccess) return e;
    {
        int first = d.mode == kModeCachedA ? 1 : 0;
        int count = d.mode == kModeProduct ? 2 : 1;
        int tiles = g.tiles;
        void* args[] = {&dd, &tt, &first, &tiles};
        e = launch(dec_kernel(g.logN1), count * g.tiles, dec_smem_bytes(), s, args);
        if (e != cudaSuccess) return e;
    }
    if (ev && (e = cudaEventRecord(ev[1], s)) != cudaSuccess) return e;
    {
        void* args[] = {&dd, &tt};
        e = launch(row_kernel(g.logN2), g.row_ctas, row_smem_bytes(), s, args);
        if (e != cudaSuccess) return e;
    }
    if (ev && (e = cudaEventRecord(ev[2], s)) != cudaSuccess) return e;
    if (d.mode != kModeForward) {
        void* args[] = {&dd, &tt};
        e = launch(crt_kernel(int(d.LW)), g.tiles, crt_smem_bytes(int(d.k)), s, args);
        if (e != cudaSuccess) return e;
    }
    if (ev && (e = cudaEventRecord(ev[3], s)) != cudaSuccess) return e;
    return cudaSuccess;
}

// ------------------------------------------------------------------ IMAD throughput probe

namespace {
constexpr int kProbeIters = 2048;
constexpr int kProbeChains = 8;

__global__ void __launch_bounds__(256) k_imad_probe(uint32_t* out, uint32_t seed) {
    uint32_t a[kProbeChains];
#pragma unroll
    for (int i = 0; i < kProbeChains; ++i) a[i] = threadIdx.x + i * 7u + seed;
    const uint32_t m = seed | 1u;
#pragma unroll 4
    for (int it = 0; it < kProbeIters; ++it) {
#pragma unroll
        for (int i = 0; i < kProbeChains; ++i) a[i] = a[i] * m + 0x9e3779b9u;
    }
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < kProbeChains; ++i) r ^= a[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}
}  // namespace

cudaError_t measure_imad_peak(double* ops_per_second) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int blocks = sms * 8, threads = 256;
    uint32_t* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if ((e = cudaMalloc(&out, size_t(blocks) * threads * 4)) != cudaSuccess) return e;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 6 && e == cudaSuccess; ++rep) {
        cudaEventRecord(e0);
        k_imad_probe<<<blocks, threads>>>(out, uint32_t(rep + 3));
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e == cudaSuccess)
        *ops_per_second = double(kProbeIters) * kProbeChains * blocks * threads / (double(best) * 1e-3);
    return e;
}

int kernels_per_product(const ProductDesc& d) { return d.mode == kModeForward ? 2 : 3; }

}  // namespace nc
