// Kernel entry points of the separately compiled kernel translation units. Each unit keeps its
// own copy of the __constant__ prime tables and uploads it in its prepare function.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "batch_types.h"
#include "common.h"

namespace nc {

// Launch with programmatic dependent launch allowed: the kernel may be scheduled once every CTA
// of the kernel before it on the stream has called pdl_trigger(), and waits for that kernel's
// results in pdl_wait() (both in arith.cuh).
inline cudaError_t launch_pdl(const void* fn, int grid, int threads, size_t smem, cudaStream_t s, void** args) {
    if (grid <= 0) return cudaSuccess;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(threads));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

void* dec_kernel(int LW);
void* dec_tc_kernel(int logN1);
void* crt_kernel(int LW);
void* crt_tc_kernel(int LW);
void* row_kernel(const RowConfig& c);
std::vector<RowConfig> all_row_variants();

cudaError_t prepare_dec(const PrimeConst* pc, const uint64_t* pow32);
cudaError_t prepare_dec_tc(const PrimeConst* pc, const uint64_t* pow32);
cudaError_t prepare_crt(const PrimeConst* pc, const uint64_t* pow32);
cudaError_t prepare_crt_tc(const PrimeConst* pc, const uint64_t* pow32);
cudaError_t prepare_row(const PrimeConst* pc, const uint64_t* pow32);
cudaError_t prepare_persistent(const PrimeConst* pc, const uint64_t* pow32);
cudaError_t prepare_residues(const PrimeConst* pc, const uint64_t* pow32);

// Residue and row items (the queue holds residue items of products on the integer residue engine).
cudaError_t launch_persistent(const BatchArgs& args, int ctas, size_t smem, cudaStream_t s);
cudaError_t launch_batch_crt(const BatchCrtArgs& args, bool tensor_cores, size_t smem, cudaStream_t s);
// Residue items of a batch on the tensor cores (BatchCrtArgs items: x = product, y = operand *
// tiles_tc + tile), every product of the launch with column length 2^logN1.
cudaError_t launch_batch_dec_tc(const BatchCrtArgs& args, int logN1, size_t smem, cudaStream_t s);
cudaError_t persistent_occupancy(size_t smem, int* ctas_per_sm);
// Row items alone, all with row blocks of 2^logN2 residues (none waits on another item).
cudaError_t launch_persistent_rows(const BatchArgs& args, int logN2, int ctas, cudaStream_t s);
cudaError_t persistent_rows_occupancy(int logN2, int* ctas_per_sm);

// The 30-bit word engine (k_w32.cu): residues of operands [first, first + count), tiles
// tile0 .. tile0 + tiles - 1 of each (128-coefficient tiles); the row stage; the CRT over
// `tiles` 256-coefficient tiles.
void* row32_kernel(const RowConfig& c);
std::vector<RowConfig> all_row32_variants();
size_t dec_tc32_smem_bytes(int k);
cudaError_t prepare_w32();
cudaError_t launch_residues32(const ProductDesc& d, const Tables& t, int logN1, cudaStream_t s, int first, int count,
                              int tile0, int tiles);
cudaError_t launch_row32(const ProductDesc& d, const Tables& t, const RowConfig& cfg, cudaStream_t s);
cudaError_t launch_crt32(const ProductDesc& d, const Tables& t, int tiles, cudaStream_t s);
// Batches on the 30-bit engine: residue items of products with column length 2^logN1 (kmax: the
// most primes among them); row items of one row-block size on `ctas` persistent CTAs; CRT items
// (lw_max: the widest LW among them, at most 30).
cudaError_t launch_batch_dec_tc32(const BatchCrtArgs& args, int logN1, int kmax, cudaStream_t s);
cudaError_t launch_persistent_rows32(const BatchArgs& args, int logN2, int ctas, cudaStream_t s);
cudaError_t persistent_rows32_occupancy(int logN2, int* ctas_per_sm);
cudaError_t launch_batch_crt_tc32(const BatchCrtArgs& args, int lw_max, cudaStream_t s);

}  // namespace nc
