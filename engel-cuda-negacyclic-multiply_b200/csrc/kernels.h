// Host-side launchers for the library's kernels.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.h"

namespace nc {

struct Tables;

// Per device: upload the __constant__ prime tables and raise the dynamic shared-memory limit of
// every kernel instantiation.
cudaError_t prepare_kernels(const PrimeConst* pc, const uint64_t* pow32);

// Row configurations with a compiled kernel that are valid for ring degree 2^logN.
std::vector<RowConfig> row_variants(int logN);
bool row_variant_exists(const RowConfig& c);

// Enqueue the three stages of one product on stream s. With `stage_events` (4 events), event i
// is recorded before stage i and event 3 after the last stage. With `b_ready` (product mode
// only), the residue stage of operand a is enqueued first and s then waits for b_ready before the
// residue stage of operand b, so a's residues overlap b's upload on another stream; b_ready
// must already be recorded.
cudaError_t launch_product(const ProductDesc& d, const Tables& t, const RowConfig& cfg, cudaStream_t s,
                           cudaEvent_t* stage_events = nullptr, cudaEvent_t b_ready = nullptr);

// Measured 32-bit IMAD throughput of this device (ops/s), from a mad.lo.u32 chain kernel.
cudaError_t measure_imad_peak(double* ops_per_second);

}  // namespace nc
