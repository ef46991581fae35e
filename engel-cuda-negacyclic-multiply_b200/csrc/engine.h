// Plans, device tables and the host-buffer pipeline behind the public entry points.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "common.h"
#include "stages.cuh"

namespace nc {

// Thrown inside the library; the C entry points turn it into a status code and message.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum : int { kOk = 0, kEInval = -1, kECuda = -2, kENoMem = -3, kETimeout = -4, kEBusy = -5 };

void check(cudaError_t e, const char* what);

// Twiddles, residue places and prime constants for every prime of the set, resident on one
// device (about 100 MB) while at least one plan on that device holds them.
struct DeviceTables {
    int device = -1;
    int refs = 0;
    ulonglong2* fwd = nullptr;
    ulonglong2* inv = nullptr;
    uint64_t* pow32 = nullptr;
    PrimeConst* pc = nullptr;
    Tables view() const { return Tables{fwd, inv, pow32, pc}; }
};

DeviceTables* acquire_tables(int device);
void release_tables(DeviceTables* t);

// Splits large host memcpys over a few worker threads.
class ParallelCopy {
  public:
    explicit ParallelCopy(int threads);
    ~ParallelCopy();
    void copy(void* dst, const void* src, size_t bytes);
    int threads() const { return int(workers_.size()) + 1; }

  private:
    void run_part(int part);
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    uint64_t gen_ = 0;
    int pending_ = 0;
    bool stop_ = false;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t bytes_ = 0;
};

// One (N, q) configuration: constants, scratch residues and staging buffers.
struct Plan {
    int device = 0;
    int N = 0, W = 0, L = 0, logN = 0, k = 0;
    QConst hq{};
    QConst* d_qc = nullptr;
    uint64_t* d_ra = nullptr;
    uint64_t* d_rb = nullptr;
    uint32_t* d_a = nullptr;
    uint32_t* d_b = nullptr;
    uint32_t* d_c = nullptr;
    uint32_t* h_a = nullptr;
    uint32_t* h_b = nullptr;
    uint32_t* h_c = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    DeviceTables* tables = nullptr;
    ParallelCopy* copier = nullptr;
    float last_kernel_ms = 0.f;
    bool timing = false;             // record per-stage events
    cudaEvent_t ev_stage[4] = {nullptr, nullptr, nullptr, nullptr};

    size_t limbs() const { return size_t(N) * size_t(L); }
    ProductDesc desc(const uint32_t* a, const uint32_t* b, uint32_t* c) const;
};

// W is the bit width the platform states for q; 0 means "take it from q".
Plan* plan_create(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q);
void plan_destroy(Plan* p);

// Device-resident product on `stream` (plan stream when null). Asynchronous.
void plan_multiply_device(Plan* p, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t stream);

// Host buffers in and out (the fherma_run contract). Synchronous.
void plan_multiply_host(Plan* p, const uint32_t* a, const uint32_t* b, uint32_t* c);

int current_device();

}  // namespace nc
