// Serving loop: continuous batching of negacyclic products under an HBM budget.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch.h"
#include "engine.h"

namespace nc {

// First-fit allocator over one region (device or pinned host), 256-byte granules.
class Arena {
  public:
    Arena() = default;
    void reset(char* base, size_t bytes);
    char* alloc(size_t bytes);  // nullptr when nothing fits
    void free(char* p);
    size_t in_use() const { return in_use_; }
    size_t capacity() const { return bytes_; }

  private:
    char* base_ = nullptr;
    size_t bytes_ = 0, in_use_ = 0;
    std::map<size_t, size_t> free_;  // offset -> size
    std::map<size_t, size_t> used_;  // offset -> size
};

// Requests carry host operands. submit() copies them into pinned staging and queues the
// request; a scheduler thread admits queued requests in arrival order as device memory (the
// HBM budget) allows, forms a batch of everything admitted, and runs it as one persistent
// launch on the next of several streams, so batches overlap on the device and new requests
// join the next batch while earlier ones run. Operands registered with register_operand()
// stay resident in their NTT-domain form and multiply later requests without being
// transformed again. wait() returns the product and the request's latency (submit to result
// in host memory).
class Server {
  public:
    Server(int device, size_t hbm_budget, size_t staging_bytes, int max_batch, int streams);
    ~Server();

    int register_operand(Plan* plan, const uint32_t* a);
    void release_operand(int id);
    uint64_t submit(Plan* plan, const uint32_t* a, int operand, const uint32_t* b);
    bool done(uint64_t id);
    double wait(uint64_t id, uint32_t* c);  // milliseconds of latency
    void stats(double* p50_ms, double* p99_ms, uint64_t* completed, double* products_per_s, size_t* hbm_in_use,
               uint64_t* batches, uint64_t* timeouts = nullptr);
    // Bytes copied host -> device and device -> host for finished batches, and on the device's clock
    // the time during which at least one batch had copies or kernels in flight (the union of the
    // batches' intervals) within the window from the first batch's start to the last one's end.
    void io_stats(uint64_t* h2d_bytes, uint64_t* d2h_bytes, double* busy_ms, double* window_ms,
                  double* scheduler_ms = nullptr);

  private:
    struct Request {
        uint64_t id;
        Plan* plan;
        int operand;
        size_t limb_bytes;
        size_t dev_bytes;
        char* host = nullptr;  // pinned: a | b | c
        char* dev = nullptr;   // device: a | b | c | scratch
        double t_submit = 0, t_done = 0;
        int status = 0;  // 0 queued, 1 in flight, 2 done, < 0 error
    };
    struct Operand {
        Plan* plan;
        char* dev;
        size_t bytes;
        int pins = 0;  // submits between their operand check and their enqueue
    };
    struct Flight {
        std::vector<Request*> reqs;
        cudaEvent_t begin = nullptr;  // before the batch's first copy
        cudaEvent_t done = nullptr;   // after its last copy
        int stream;
        uint64_t h2d = 0, d2h = 0;
    };

    void loop();
    void launch(std::vector<Request*>& reqs);
    bool reap(bool block);

    int device_;
    int max_batch_;
    char* dev_base_ = nullptr;
    char* host_base_ = nullptr;
    Arena dev_arena_, host_arena_;
    std::vector<cudaStream_t> streams_;
    std::vector<std::unique_ptr<Batch>> batches_;
    std::vector<bool> stream_busy_;
    int next_stream_ = 0;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_, space_cv_;
    std::deque<Request*> queue_;
    std::deque<Flight> flights_;
    std::map<uint64_t, std::unique_ptr<Request>> requests_;
    std::map<int, Operand> operands_;
    int next_operand_ = 0;
    uint64_t next_id_ = 1;
    bool stop_ = false;
    std::string fault_;
    std::vector<double> latencies_;
    double t_first_ = -1, t_last_ = 0;
    uint64_t batches_run_ = 0;
    uint64_t timeouts_ = 0;  // batches whose dependency wait gave up (their requests fail)
    cudaEvent_t origin_ = nullptr;                    // device-clock origin of the batch intervals
    std::vector<std::pair<double, double>> busy_;    // [begin, end) of finished batches, ms from origin_
    uint64_t h2d_bytes_ = 0, d2h_bytes_ = 0;
    double launch_ms_ = 0;  // host time the scheduler thread spent enqueueing batches
    std::string last_timeout_;  // what the last such wait waited for
    std::thread thread_;
};

}  // namespace nc
