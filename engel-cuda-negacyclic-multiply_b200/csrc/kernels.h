// Host-side launchers for the plain per-call kernels.
#pragma once

#include <cuda_runtime.h>

#include "common.h"

namespace nc {

struct Tables;

// Raise the dynamic shared-memory limit of every kernel instantiation (once per device).
cudaError_t prepare_plain_kernels();

// Enqueue the three stages of one product on stream s. With `stage_events` (4 events), event i
// is recorded before stage i and event 3 after the last stage.
cudaError_t launch_product(const ProductDesc& d, const Tables& t, cudaStream_t s,
                           cudaEvent_t* stage_events = nullptr);

// Measured 32-bit IMAD throughput of this device (ops/s), from a mad.lo.u32 chain kernel.
cudaError_t measure_imad_peak(double* ops_per_second);

// Kernel launches that launch_product issues for this descriptor.
int kernels_per_product(const ProductDesc& d);

}  // namespace nc
