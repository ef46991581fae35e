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

// Residue tiles per operand of the product's residue engine (each covers a run of columns of
// every row segment: the tiles of group g out of G cover columns [g N2 / G, (g + 1) N2 / G)).
int residue_tiles(const ProductDesc& d, const RowConfig& cfg);

// Enqueue the residue stage (with the forward column stages) of operands [first, first + count)
// of the product on stream s: the tiles of group `group` out of `groups` (all of them by default;
// `groups` must divide residue_tiles).
cudaError_t launch_residues(const ProductDesc& d, const Tables& t, const RowConfig& cfg, cudaStream_t s, int first,
                            int count, int group = 0, int groups = 1);

// Enqueue the three stages of one product on stream s. With `stage_events` (4 events), event i
// is recorded before stage i and event 3 after the last stage. With `b_ready` (product and
// cached-a modes), operand a must already be taken care of on s (product: its residue stage,
// launch_residues(d, .., 0, 1); cached-a: a forward-mode launch that wrote d.a_hat), with stage
// event 0 recorded before that by the caller: s waits for b_ready, then runs the residue stage
// of the other operands, so a's stages overlap their upload on another stream. b_ready must
// already be recorded.
// With `residues_done`, every operand's residue stage is already enqueued on s, and only the row
// and CRT stages are (b_ready is then ignored).
cudaError_t launch_product(const ProductDesc& d, const Tables& t, const RowConfig& cfg, cudaStream_t s,
                           cudaEvent_t* stage_events = nullptr, cudaEvent_t b_ready = nullptr,
                           bool residues_done = false);

// Per device, with that device current: look up (and so load onto the device) the fixed scratch
// array of the allocation-free entry point. Called once when the device's tables are set up.
cudaError_t prepare_noalloc(int device);

// Measured 32-bit IMAD throughput of this device (ops/s), from a mad.lo.u32 chain kernel.
cudaError_t measure_imad_peak(double* ops_per_second);

}  // namespace nc
