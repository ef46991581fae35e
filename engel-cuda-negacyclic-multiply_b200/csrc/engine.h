// Plans, device tables and the host-buffer pipeline behind the public entry points.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "common.h"

namespace nc {

// Thrown inside the library; the C entry points turn it into a status code and message.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum : int { kOk = 0, kEInval = -1, kECuda = -2, kENoMem = -3, kETimeout = -4, kEBusy = -5, kESelfCheck = -6 };

void check(cudaError_t e, const char* what);

// Twiddles, residue places and prime constants for every prime of the set, resident on one
// device (about 100 MB) while at least one plan on that device holds them.
struct DeviceTables {
    int device = -1;
    int refs = 0;
    ulonglong2* fwd = nullptr;
    ulonglong2* inv = nullptr;
    uint64_t* pow32 = nullptr;   // [kMaxPrimes][kMaxL]
    uint64_t* primes = nullptr;  // [kMaxPrimes]
    uint4* res_w = nullptr;      // weight bytes of the tensor-core residue stage
    bool tensor_cores = false;   // compute capability 10.0: the sm_100a tcgen05 kernels run here
    // the 30-bit word engine's tables (about 75 MB; only on devices with tensor cores)
    uint2* fwd32 = nullptr;
    uint2* inv32 = nullptr;
    PrimeConst32* pc32 = nullptr;
    uint32_t* pow32_32 = nullptr;
    uint4* res_w32 = nullptr;
    Tables view() const { return Tables{fwd, inv, pow32, primes, res_w, fwd32, inv32, pc32, pow32_32, res_w32}; }
};

// Known answers of the host arithmetic, the prime set and sampled tables, checked once per
// process ("" when they hold).
const std::string& host_self_check();

// An N = 8 product on `device` against the host schoolbook, once per device (the first plan
// created there runs it); throws Error(kESelfCheck) on a mismatch.
void device_self_test(int device);

DeviceTables* acquire_tables(int device);
void release_tables(DeviceTables* t);

// A few host worker threads that run one job at a time, every thread (workers and the caller)
// on its own part. Workers spin briefly between jobs, so the back-to-back jobs of one product
// hand over in microseconds, then sleep.
class HostPool {
  public:
    explicit HostPool(int threads);
    ~HostPool();
    int parts() const { return int(workers_.size()) + 1; }
    // fn(part, parts) on every thread; returns when all parts are done.
    void run(const std::function<void(int, int)>& fn);

  private:
    void worker(int part);
    std::vector<std::thread> workers_;
    std::mutex run_mu_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::atomic<uint64_t> gen_{0};
    std::atomic<int> pending_{0};
    std::atomic<bool> stop_{false};
    const std::function<void(int, int)>* job_ = nullptr;
};

// Device-to-host copies (and events) of one product on the host path, at most.
constexpr int kMaxOutChunks = 16;

// One (N, q) configuration: constants, scratch residues and staging buffers.
struct Plan {
    int device = 0;
    int N = 0, W = 0, L = 0, logN = 0, k = 0;
    QConst hq{};
    QConst* d_qc = nullptr;
    uint64_t* d_ra = nullptr;
    uint64_t* d_rb = nullptr;
    int factors = 2;                                    // operands the plan's primes cover
    uint64_t* d_rx[kMaxFactors - 2] = {};               // residues of operands 3, 4 (chained plans)
    uint32_t* d_x[kMaxFactors - 2] = {};                // host path: device copies of operands 3, 4
    uint32_t* h_x[kMaxFactors - 2] = {};                // host path: pinned staging of operands 3, 4
    uint32_t* d_a = nullptr;
    uint32_t* d_b = nullptr;
    uint32_t* d_c = nullptr;
    uint32_t* h_a = nullptr;
    uint32_t* h_b = nullptr;
    uint32_t* h_c = nullptr;
    uint64_t* d_hat = nullptr;  // host path: NTT form of operand a (k x N), made while b uploads
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    std::vector<cudaEvent_t> ev_out;  // one per output chunk
    std::vector<cudaEvent_t> ev_grp;  // host path: a column group of operand b has landed
    cudaStream_t copy_stream = nullptr;         // host path: operand b's upload
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;  // operand a uploaded / operand b uploaded
    DeviceTables* tables = nullptr;
    HostPool* pool = nullptr;
    float last_kernel_ms = 0.f;
    RowConfig cfg{};                 // row-stage tiling of the plain path (autotuned per N)
    uint4* d_crt_b = nullptr;        // byte table of the tensor-core CRT (k <= 32), built at creation
    bool crt_tc = true;              // plain path: CRT accumulation on the tensor cores when available
    bool res_tc = true;              // plain path: residue stage on the tensor cores
    // The 30-bit word engine for the plain path of a pair (k32 primes below 2^30): available with
    // tensor cores when the bound fits 64 primes; in use while `w32` is set and both tensor-core
    // stages are selected. Batches, chains and the allocation-free entry run the 62-bit engine.
    bool w32_ok = false;
    bool w32 = false;
    int k32 = 0;
    QConst32 hq32{};
    QConst32* d_qc32 = nullptr;
    uint4* d_crt_b32 = nullptr;
    RowConfig cfg32{};               // row-stage tiling of the 30-bit engine
    bool timing = false;             // record per-stage events
    cudaEvent_t ev_stage[4] = {nullptr, nullptr, nullptr, nullptr};
    // Host-path trace (NC_TRACE=1 in the environment when the plan is created): every host-buffer
    // product writes one line to stderr with its phases in microseconds since the call began.
    bool trace = false;
    cudaEvent_t ev_trace[6] = {};  // call start, a uploaded, a forward, b uploaded, product, downloaded
    double trace_host[4] = {0, 0, 0, 0};  // a staged, b staged, enqueued, collected (us)
    std::chrono::steady_clock::time_point trace_t0;

    size_t limbs() const { return size_t(N) * size_t(L); }
    bool use_w32() const { return w32 && w32_ok && res_tc && crt_tc; }
    // Row configuration and descriptor of the plain path's engine.
    const RowConfig& plain_cfg() const { return use_w32() ? cfg32 : cfg; }
    ProductDesc desc_plain(const uint32_t* a, const uint32_t* b, uint32_t* c) const;
    // Bytes of one operand's residue scratch (either engine).
    size_t residue_bytes() const;
    // The 62-bit engine's descriptor.
    ProductDesc desc(const uint32_t* a, const uint32_t* b, uint32_t* c) const;
    // All `factors` operands of a chained product (device pointers).
    ProductDesc desc_chain(const uint32_t* const* x, uint32_t* c) const;
};

// W is the bit width the platform states for q; 0 means "take it from q". `factors` (2 to 4) is
// the number of operands one product multiplies: the prime count covers the bound of that many.
Plan* plan_create(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int factors = 2);
void plan_destroy(Plan* p);

// Plain-path resources, allocated on first use (cheap plans for batches and servers).
void ensure_scratch(Plan* p);
void ensure_host_path(Plan* p);

// Device-resident product on `stream` (0: the CUDA default stream). Asynchronous.
void plan_multiply_device(Plan* p, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t stream);
// Chained product of the plan's `factors` device operands x[0..factors): one residue stage per
// operand, every forward transform and pointwise product, one inverse transform, one CRT.
void plan_multiply_chain_device(Plan* p, const uint32_t* const* d_x, uint32_t* d_c, cudaStream_t stream);

// Host buffers in and out (the fherma_run contract), in two halves so a caller can do host work
// while the GPU computes. submit: every pool thread stages a slice of a and b into pinned memory
// and enqueues that slice's H2D copy (memcpy and DMA overlap), then the kernels and the chunked
// D2H are enqueued. collect: each pool thread waits for its output chunk and copies it out.
void plan_submit_host(Plan* p, const uint32_t* a, const uint32_t* b);
void plan_collect_host(Plan* p, uint32_t* c);
void plan_multiply_host(Plan* p, const uint32_t* a, const uint32_t* b, uint32_t* c);
// The chained product with host operands x[0..factors) (same staging as the pair).
void plan_multiply_chain_host(Plan* p, const uint32_t* const* x, uint32_t* c);

int current_device();

// Row configuration for the plain path of a plan: validated and applied.
void plan_set_row_config(Plan* p, const RowConfig& c);

// Times every compiled row configuration valid for the plan's N on its own buffers (`reps`
// products each, device-resident), applies the fastest and remembers it for later plans of
// the same (N, L). Returns the best device milliseconds per product.
float plan_autotune(Plan* p, int reps);

// The remembered choice for (logN, L), if any autotune ran in this process.
bool tuned_row_config(int logN, int L, RowConfig* out);
// The 30-bit engine's remembered row configuration for (logN, L) and whether it was the faster.
bool tuned_engine(int logN, int L, RowConfig* cfg32, bool* use_w32);

// The plain path's engine: 32 (the 30-bit word engine; throws if the plan cannot run it) or 64.
void plan_set_word_bits(Plan* p, int bits);

}  // namespace nc
