// Host-side dispatch of the kernels: which instantiation runs a product, per-device preparation,
// and the IMAD throughput probe.
#include <cuda_runtime.h>

#include "kernel_registry.h"
#include "kernels.h"

namespace nc {

namespace {

// The product kernels go out with programmatic dependent launch: each may be scheduled while the
// kernel before it on the stream finishes its last wave (see pdl_wait / pdl_trigger).
cudaError_t launch(void* fn, int grid, int threads, size_t smem, cudaStream_t s, void** args) {
    return launch_pdl(fn, grid, threads, smem, s, args);
}

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

bool row_variant_exists(const RowConfig& c) { return row_kernel(c) != nullptr; }

std::vector<RowConfig> row_variants(int logN) {
    std::vector<RowConfig> out;
    for (const RowConfig& c : all_row_variants())
        if (row_config_valid(logN, c)) out.push_back(c);
    return out;
}

cudaError_t prepare_kernels(const PrimeConst* pc, const uint64_t* pow32) {
    cudaError_t e = prepare_dec(pc, pow32);
    if (e == cudaSuccess) e = prepare_dec_tc(pc, pow32);
    if (e == cudaSuccess) e = prepare_row(pc, pow32);
    if (e == cudaSuccess) e = prepare_crt(pc, pow32);
    if (e == cudaSuccess) e = prepare_crt_tc(pc, pow32);
    if (e == cudaSuccess) e = prepare_persistent(pc, pow32);
    if (e == cudaSuccess) e = prepare_residues(pc, pow32);
    if (e == cudaSuccess) e = prepare_w32();
    return e;
}

int residue_tiles(const ProductDesc& d, const RowConfig& cfg) {
    if (d.res_tc) {
        const int n = 1 << d.logN;
        return n < kDecTcRows ? 1 : n / kDecTcRows;
    }
    return geometry(int(d.logN), int(d.k), cfg).tiles;
}

cudaError_t launch_residues(const ProductDesc& d, const Tables& t, const RowConfig& cfg, cudaStream_t s, int first,
                            int count, int group, int groups) {
    ProductDesc dd = d;
    Tables tt = t;
    if (d.res_tc && !t.res_w) return cudaErrorInvalidValue;
    const int all = residue_tiles(d, cfg);
    if (groups < 1 || group < 0 || group >= groups || all % groups != 0) return cudaErrorInvalidValue;
    int tiles = all / groups;
    int tile0 = group * tiles;
    if (d.qc32) return launch_residues32(d, t, int(d.logN) - cfg.logN2, s, first, count, tile0, tiles);
    void* args[] = {&dd, &tt, &first, &tile0, &tiles};
    if (d.res_tc) {
        // tensor-core residues: 128-coefficient tiles
        void* dec = dec_tc_kernel(int(d.logN) - cfg.logN2);
        if (!dec) return cudaErrorInvalidValue;
        return launch(dec, count * tiles, kThreads, dec_tc_smem_bytes(int(d.k)), s, args);
    }
    void* dec = dec_kernel(int(d.LW));
    if (!dec) return cudaErrorInvalidValue;
    return launch(dec, count * tiles, kThreads, dec_smem_bytes(int(d.k)), s, args);
}

cudaError_t launch_product(const ProductDesc& d, const Tables& t, const RowConfig& cfg, cudaStream_t s,
                           cudaEvent_t* ev, cudaEvent_t b_ready, bool residues_done) {
    if (int(d.logN2) != cfg.logN2) return cudaErrorInvalidValue;
    const bool w32 = d.qc32 != nullptr;
    void* row = w32 ? row32_kernel(cfg) : row_kernel(cfg);
    void* crt = d.crt_b ? crt_tc_kernel(int(d.LW)) : crt_kernel(int(d.LW));
    if (!row || !crt || !dec_kernel(int(d.LW))) return cudaErrorInvalidValue;
    if (w32 && d.factors != 2) return cudaErrorInvalidValue;  // the 30-bit engine multiplies pairs
    const Geometry g = geometry(int(d.logN), int(d.k), cfg);
    ProductDesc dd = d;
    Tables tt = t;
    cudaError_t e;
    const int factors = d.mode == kModeProduct ? int(d.factors) : 1;
    if (residues_done) {
        // every operand's residue stage is already on s (the host path's grouped upload)
    } else if (b_ready && d.mode != kModeForward) {
        // operand a is already taken care of on s (its residues, or its NTT form for a cached-a
        // product); the other operands follow once they have landed
        if ((e = cudaStreamWaitEvent(s, b_ready, 0)) != cudaSuccess) return e;
        const int rest = d.mode == kModeProduct ? factors - 1 : 1;
        if ((e = launch_residues(d, t, cfg, s, 1, rest)) != cudaSuccess) return e;
    } else {
        if (ev && (e = cudaEventRecord(ev[0], s)) != cudaSuccess) return e;
        const int first = d.mode == kModeCachedA ? 1 : 0;
        if ((e = launch_residues(d, t, cfg, s, first, factors)) != cudaSuccess) return e;
    }
    if (ev && (e = cudaEventRecord(ev[1], s)) != cudaSuccess) return e;
    if (w32) {
        e = launch_row32(d, t, cfg, s);
    } else {
        void* args[] = {&dd, &tt};
        e = launch(row, g.row_ctas, cfg.threads, row_smem_bytes(cfg.threads, cfg.logE), s, args);
    }
    if (e != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[2], s)) != cudaSuccess) return e;
    if (d.mode != kModeForward) {
        if (w32) {
            e = launch_crt32(d, t, g.tiles, s);
        } else {
            void* args[] = {&dd, &tt};
            e = launch(crt, g.tiles, kThreads, d.crt_b ? crt_tc_smem_bytes(int(d.LW)) : crt_smem_bytes(int(d.k)), s,
                       args);
        }
        if (e != cudaSuccess) return e;
    }
    if (ev && (e = cudaEventRecord(ev[3], s)) != cudaSuccess) return e;
    return cudaSuccess;
}

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

}  // namespace nc
