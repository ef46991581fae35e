// Batches of products: one persistent launch for residues and rows, then the CRT launches (host side).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

namespace nc {


// A list of products (each referring to a plan for its q, N and constants) that run together.
// Products may differ in N and in q. Residue scratch comes from the batch's own arena. A run is,
// for products below N = 2^15: the tensor-core residue launches, one persistent launch for the
// row stage (and any residue items on the integer pipes), then one CRT launch per CRT engine in
// use. Products of N >= 2^15 fill the GPU on their own: they run the plain path's launches with
// their plan's row configuration, alternating between two streams so that one product's last
// wave overlaps the next one's kernels. Plain products (a, b -> c) of plans on the 30-bit word
// engine run on it (residue scratch from the batch's arena): below 2^15 in their own residue,
// persistent-row and CRT launches after the 62-bit ones, from 2^15 as the plain path's launches.
// The counter reset and the launches are captured once into a CUDA graph and replayed while the
// batch keeps the same shape.
class Batch {
  public:
    explicit Batch(int device);
    ~Batch();

    // mode: kModeProduct (a, b -> c), kModeCachedA (a_hat in the NTT domain, b -> c),
    //       kModeForward (a -> a_hat: the NTT-domain form of an operand, for caching).
    // `scratch` (optional): 2 * k * N u64 of residue scratch owned by the caller; without it the
    // product takes its scratch from the batch's own arena.
    void add(Plan* plan, uint32_t mode, const uint32_t* a, const uint32_t* b, uint32_t* c, const uint64_t* a_hat,
             uint64_t* hat_out, uint64_t* scratch = nullptr);
    void clear();
    size_t size() const { return entries_.size(); }
    // Enqueue the whole batch on `stream` (graph replay when `use_graph`).
    void run(cudaStream_t stream, bool use_graph);
    // Wait for the last run and check that no dependency wait gave up.
    void synchronize();
    int ctas() const { return ctas_; }
    size_t scratch_bytes() const { return scratch_bytes_; }
    int launches_per_run() const {
        int n = (n_items_ > 0 ? (with_dec_ ? 1 : int(row_groups_.size())) : 0) + (n_crt_tc_ > 0 ? 1 : 0) +
                (n_crt_ > 0 ? 1 : 0);
        for (int c : n_dec_tc_) n += c > 0 ? 1 : 0;
        for (const Direct& x : direct_) n += x.d.mode == kModeForward ? 2 : 3;
        n += int(row_groups32_.size()) + (n_crt_tc32_ > 0 ? 1 : 0);
        for (int c : n_dec_tc32_) n += c > 0 ? 1 : 0;
        return n;
    }
    // After the last run has completed (its event): did a dependency wait give up?
    bool failed() const;
    // What the failed wait waited for (empty when nothing failed).
    std::string failure() const;

  private:
    struct Entry {
        Plan* plan;
        uint32_t mode;
        const uint32_t* a;
        const uint32_t* b;
        uint32_t* c;
        const uint64_t* a_hat;
        uint64_t* hat_out;
        uint64_t* scratch;
    };
    // A product of N >= 2^15, launched as on the plain path.
    struct Direct {
        ProductDesc d;
        RowConfig cfg;
    };
    static constexpr int kDirectLogN = 15;
    // Without residue items in the queue, the row items go by row-block size, one persistent
    // launch each (k_persistent_rows<logN2>): items [first, first + count) of the queue.
    struct RowGroup {
        int logN2, first, count, ctas;
    };
    std::vector<RowGroup> row_groups_;
    void finalize(cudaStream_t stream);
    int device_;
    std::vector<Direct> direct_;
    cudaStream_t side_ = nullptr;                    // second stream of the direct products
    cudaEvent_t fork_ = nullptr, join_ = nullptr;
    std::vector<Entry> entries_;
    std::vector<uint64_t> shape_;  // signature of the captured graph
    DeviceTables* tables_ = nullptr;
    void* d_products_ = nullptr;
    size_t products_cap_ = 0;
    uint2* d_items_ = nullptr;
    size_t items_cap_ = 0;
    uint32_t* d_state_ = nullptr;  // counters (2 per product), head, error[4], a head per row group
    size_t state_cap_ = 0;
    char* h_upload_ = nullptr;  // pinned: product table | item list, copied on the run's stream
    size_t h_upload_cap_ = 0;
    uint64_t* scratch_ = nullptr;
    size_t scratch_bytes_ = 0;
    int n_items_ = 0;
    int ctas_ = 0;
    size_t smem_ = 0;      // persistent launch (row items, and residue items on the integer pipes)
    bool with_dec_ = false;  // the persistent queue holds residue items
    int n_crt_tc_ = 0;     // CRT items on the tensor cores, after the persistent queue in d_items_
    int n_crt_ = 0;        // CRT items on the integer pipes, after those
    size_t smem_crt_tc_ = 0, smem_crt_ = 0;
    int n_dec_tc_[kMaxLogN1 + 1] = {};  // tensor-core residue items by log2 N1, after the CRT items
    size_t smem_dec_tc_ = 0;
    // Products on the 30-bit engine (plain products of plans that use it, residue scratch from the
    // batch's arena), after the items above in d_items_: their row items by row-block size (one
    // persistent launch each; heads after the 62-bit groups'), their CRT items, their residue items
    // by log2 N1.
    std::vector<RowGroup> row_groups32_;
    int n_crt_tc32_ = 0;
    int n_dec_tc32_[kMaxLogN1 + 1] = {};
    int crt32_first_ = 0, dec32_first_ = 0;  // positions in d_items_
    int kmax32_ = 1, lw_tc32_ = 2;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaEvent_t done_ = nullptr;  // recorded after every run
    bool ran_ = false;
    bool dirty_ = true;
    uint32_t* err_host_ = nullptr;  // pinned copy of the run's error flag, written before done_
};

}  // namespace nc
