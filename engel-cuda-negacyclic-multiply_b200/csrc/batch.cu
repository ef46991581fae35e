// Batches of products: one persistent launch for residues and rows, then the CRT launches (host side).
#include "batch.h"

#include <algorithm>
#include <cstring>

#include "batch_types.h"
#include "kernel_registry.h"
#include "kernels.h"

namespace nc {

namespace {

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <class T>
void ensure(T** p, size_t* cap, size_t count, const char* what) {
    if (count <= *cap && *p) return;
    cudaFree(*p);
    *p = nullptr;
    const size_t n = std::max<size_t>(count, 1) * 2;
    check(cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)), what);
    *cap = n;
}

}  // namespace

Batch::Batch(int device) : device_(device) {
    tables_ = acquire_tables(device);
    cudaError_t e = cudaEventCreateWithFlags(&done_, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join_, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&err_host_, 4 * sizeof(uint32_t));
    if (e != cudaSuccess) {
        if (done_) cudaEventDestroy(done_);
        if (fork_) cudaEventDestroy(fork_);
        if (join_) cudaEventDestroy(join_);
        if (side_) cudaStreamDestroy(side_);
        release_tables(tables_);
        check(e, "batch event");
    }
    *err_host_ = 0;
}

bool Batch::failed() const { return ran_ && *err_host_ != 0; }

Batch::~Batch() {
    // wait on the batch's own event (never on the caller's stream, which may be gone)
    if (ran_) cudaEventSynchronize(done_);
    cudaEventDestroy(done_);
    cudaEventDestroy(fork_);
    cudaEventDestroy(join_);
    cudaStreamDestroy(side_);
    cudaFreeHost(err_host_);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    cudaFree(d_products_);
    cudaFree(d_items_);
    cudaFree(d_state_);
    cudaFreeHost(h_upload_);
    cudaFree(scratch_);
    release_tables(tables_);
}

void Batch::add(Plan* plan, uint32_t mode, const uint32_t* a, const uint32_t* b, uint32_t* c, const uint64_t* a_hat,
                uint64_t* hat_out, uint64_t* scratch) {
    if (!plan) throw Error(kEInval, "null plan");
    if (plan->device != device_) throw Error(kEInval, "the plan lives on another device");
    if (mode > kModeForward) throw Error(kEInval, "unknown product mode");
    const bool need_a = mode != kModeCachedA, need_b = mode != kModeForward;
    if ((need_a && !a) || (need_b && (!b || !c)) || (mode == kModeCachedA && !a_hat) ||
        (mode == kModeForward && !hat_out))
        throw Error(kEInval, "missing device buffer for this product mode");
    const uintptr_t align = reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
                            reinterpret_cast<uintptr_t>(c) | reinterpret_cast<uintptr_t>(a_hat) |
                            reinterpret_cast<uintptr_t>(hat_out);
    if (align & 15) throw Error(kEInval, "device buffers must be 16-byte aligned");
    if (entries_.size() >= (size_t(1) << 28)) throw Error(kEInval, "batch too large");
    if (reinterpret_cast<uintptr_t>(scratch) & 255) throw Error(kEInval, "scratch must be 256-byte aligned");
    entries_.push_back(Entry{plan, mode, a, b, c, a_hat, hat_out, scratch});
    dirty_ = true;
}

void Batch::clear() {
    entries_.clear();
    dirty_ = true;
}

void Batch::finalize(cudaStream_t stream) {
    // the previous run may still read the device-side product and item tables
    if (ran_) check(cudaEventSynchronize(done_), "batch");
    const size_t n = entries_.size();
    std::vector<BatchProduct> prods(n);
    std::vector<uint64_t> shape;
    size_t scratch = 0;
    int kmax = 1, kmax_imad = 0, kmax_tc = 0;
    // every entry of a plan that runs the 30-bit engine runs it here too (its NTT-domain operands
    // are 30-bit residues, and caller scratch holds Plan::residue_bytes, enough for either engine)
    auto on_w32 = [](const Entry& e) { return e.plan->use_w32(); };
    auto residue_bytes = [&](const Entry& e) {
        return round_up(on_w32(e) ? e.plan->residue_bytes() : size_t(e.plan->k) * e.plan->N * sizeof(uint64_t), 256);
    };
    for (size_t p = 0; p < n; ++p) {
        const Plan* pl = entries_[p].plan;
        if (!entries_[p].scratch) scratch += 2 * residue_bytes(entries_[p]);
        kmax = std::max(kmax, pl->k);
        (pl->res_tc ? kmax_tc : kmax_imad) = std::max(pl->res_tc ? kmax_tc : kmax_imad, pl->k);
    }
    if (scratch > scratch_bytes_) {
        cudaFree(scratch_);
        scratch_ = nullptr;
        scratch_bytes_ = 0;
        check(cudaMalloc(&scratch_, scratch), "batch scratch");
        scratch_bytes_ = scratch;
    }
    std::vector<uint2> dec, row, crt, crt_tc, dec_tc[kMaxLogN1 + 1];
    std::vector<uint2> row_by_size[kBatchRowLogMax + 1];
    std::vector<uint2> crt_tc32, dec_tc32[kMaxLogN1 + 1], row32_by_size[kBatchRowLogMax + 1],
        row32_tail[kBatchRowLogMax + 1];
    kmax32_ = 1;
    lw_tc32_ = 2;
    direct_.clear();
    int lw_tc = 2;
    size_t off = 0;
    char* base = reinterpret_cast<char*>(scratch_);
    for (size_t p = 0; p < n; ++p) {
        const Entry& e = entries_[p];
        const Plan* pl = e.plan;
        const RowConfig cfg = batch_row_config(pl->logN);
        const Geometry g = geometry(pl->logN, pl->k, cfg);
        ProductDesc d = pl->desc(e.a, e.b, e.c);
        d.logN2 = uint32_t(cfg.logN2);
        d.mode = e.mode;
        d.a_hat = e.a_hat;
        d.hat_out = e.hat_out;
        const size_t res = residue_bytes(e);
        if (e.scratch) {
            d.ra = e.scratch;
            d.rb = e.scratch + res / sizeof(uint64_t);
        } else {
            d.ra = reinterpret_cast<uint64_t*>(base + off);
            d.rb = reinterpret_cast<uint64_t*>(base + off + res);
            off += 2 * res;
        }
        if (pl->logN >= kDirectLogN) {
            // fills the GPU alone: the plain path's launches with the plan's row configuration
            const bool w32 = on_w32(e);
            const RowConfig& dc = w32 ? pl->cfg32 : pl->cfg;
            if (w32) {
                ProductDesc dw = pl->desc_plain(e.a, e.b, e.c);
                dw.ra = d.ra;
                dw.rb = d.rb;
                dw.mode = e.mode;
                dw.a_hat = e.a_hat;
                dw.hat_out = e.hat_out;
                d = dw;
            }
            d.logN2 = uint32_t(dc.logN2);
            direct_.push_back(Direct{d, dc});
            shape.push_back((uint64_t(1) << 63) | (uint64_t(w32) << 62) | (uint64_t(pl->logN) << 40) |
                            (uint64_t(d.k) << 32) | (uint64_t(dc.logN2) << 24) | (uint64_t(dc.logE) << 16) |
                            (uint64_t(dc.threads) << 4) | e.mode);
            continue;
        }
        BatchProduct& bp = prods[p];
        if (on_w32(e)) {
            // the 30-bit engine: residue items on the tensor cores, row items by block size, CRT items
            const Geometry g32 = geometry(pl->logN, pl->k32, cfg);
            ProductDesc dw = pl->desc_plain(e.a, e.b, e.c);
            dw.ra = d.ra;
            dw.rb = d.rb;
            dw.logN2 = uint32_t(cfg.logN2);
            dw.mode = e.mode;
            dw.a_hat = e.a_hat;
            dw.hat_out = e.hat_out;
            bp.d = dw;
            bp.tiles = uint32_t(g32.tiles);
            // operands with a residue stage: both (product), a (forward) or b (cached a)
            bp.first_operand = e.mode == kModeCachedA ? 1u : 0u;
            const uint32_t operands = e.mode == kModeProduct ? 2u : 1u;
            bp.tiles_tc = uint32_t(pl->N < kDecTcRows ? 1 : pl->N / kDecTcRows);
            bp.n_dec = 0;
            bp.n_row = uint32_t(g32.row_ctas);
            const uint32_t pid = uint32_t(p);
            for (uint32_t i = 0; i < operands * bp.tiles_tc; ++i) dec_tc32[g32.logN1].push_back(make_uint2(pid, i));
            const int logN1_32 = pl->logN - cfg.logN2;
            if (e.mode == kModeProduct && cfg.logN2 == kBatchRowLogMax && logN1_32 >= 1) {
                // row pairs (k_persistent_rows32 takes two adjacent items): row blocks u and
                // N1 - 1 - u of each prime next to each other, an even count per product
                const uint32_t n1 = 1u << logN1_32;
                for (uint32_t i = 0; i < uint32_t(pl->k32); ++i)
                    for (uint32_t u = 0; u < n1 / 2; ++u) {
                        row32_by_size[cfg.logN2].push_back(make_uint2((kItemRow << 28) | pid, i * n1 + u));
                        row32_by_size[cfg.logN2].push_back(make_uint2((kItemRow << 28) | pid, i * n1 + n1 - 1 - u));
                    }
            } else {
                // after every product's pairs, so that the pairs stay aligned to even positions
                for (uint32_t i = 0; i < bp.n_row; ++i) row32_tail[cfg.logN2].push_back(make_uint2((kItemRow << 28) | pid, i));
            }
            if (e.mode != kModeForward)
                for (uint32_t i = 0; i < uint32_t(g32.tiles); ++i) crt_tc32.push_back(make_uint2(pid, i));
            kmax32_ = std::max(kmax32_, pl->k32);
            lw_tc32_ = std::max(lw_tc32_, int(dw.LW));
            shape.push_back((uint64_t(1) << 61) | (uint64_t(pl->logN) << 40) | (uint64_t(pl->k32) << 32) |
                            (uint64_t(pl->L) << 8) | e.mode);
            continue;
        }
        bp.d = d;
        bp.tiles = uint32_t(g.tiles);
        bp.first_operand = e.mode == kModeCachedA ? 1u : 0u;
        bp.tiles_tc = uint32_t(pl->N < kDecTcRows ? 1 : pl->N / kDecTcRows);
        const uint32_t operands = e.mode == kModeProduct ? 2u : 1u;
        const uint32_t pid = uint32_t(p);
        if (d.res_tc) {
            // residues on the tensor cores, in a launch before the persistent one: the product's row
            // items then wait for no residue item
            bp.n_dec = 0;
            for (uint32_t i = 0; i < operands * bp.tiles_tc; ++i) dec_tc[g.logN1].push_back(make_uint2(pid, i));
        } else {
            bp.n_dec = operands * uint32_t(g.tiles);
        }
        bp.n_row = uint32_t(g.row_ctas);
        for (uint32_t i = 0; i < bp.n_dec; ++i) dec.push_back(make_uint2((kItemDec << 28) | pid, i));
        for (uint32_t i = 0; i < bp.n_row; ++i) {
            row.push_back(make_uint2((kItemRow << 28) | pid, i));
            row_by_size[cfg.logN2].push_back(make_uint2((kItemRow << 28) | pid, i));
        }
        if (e.mode != kModeForward) {
            // CRT on the tensor cores for products with a table and at most 30 limbs
            const bool tc = d.crt_b && crt_tc_tmem_cols(int(d.LW)) == 256;
            if (tc) lw_tc = std::max(lw_tc, int(d.LW));
            for (uint32_t i = 0; i < uint32_t(g.tiles); ++i) (tc ? crt_tc : crt).push_back(make_uint2(pid, i));
        }
        shape.push_back((uint64_t(pl->logN) << 40) | (uint64_t(pl->k) << 32) | (uint64_t(pl->L) << 8) | e.mode);
    }
    // queue of the persistent launch (residue, then row items; without residue items, the row
    // items grouped by row-block size, one launch per group), then the two CRT item lists
    with_dec_ = !dec.empty();
    std::vector<uint2> items;
    items.reserve(dec.size() + row.size() + crt_tc.size() + crt.size());
    row_groups_.clear();
    if (with_dec_) {
        items.insert(items.end(), dec.begin(), dec.end());
        items.insert(items.end(), row.begin(), row.end());
    } else {
        for (int l = kBatchRowLogMax; l >= 1; --l) {
            if (row_by_size[l].empty()) continue;
            row_groups_.push_back(RowGroup{l, int(items.size()), int(row_by_size[l].size()), 0});
            items.insert(items.end(), row_by_size[l].begin(), row_by_size[l].end());
            shape.push_back((uint64_t(3) << 60) | (uint64_t(l) << 32) | uint64_t(row_by_size[l].size()));
        }
    }
    n_items_ = int(items.size());
    n_crt_tc_ = int(crt_tc.size());
    n_crt_ = int(crt.size());
    items.insert(items.end(), crt_tc.begin(), crt_tc.end());
    items.insert(items.end(), crt.begin(), crt.end());
    shape.push_back((uint64_t(n_crt_tc_) << 32) | uint64_t(lw_tc));
    for (int l = 0; l <= kMaxLogN1; ++l) {
        n_dec_tc_[l] = int(dec_tc[l].size());
        items.insert(items.end(), dec_tc[l].begin(), dec_tc[l].end());
        shape.push_back((uint64_t(l) << 32) | uint64_t(n_dec_tc_[l]));
    }
    shape.push_back(uint64_t(kmax_tc));
    // the 30-bit products' items
    row_groups32_.clear();
    for (int l = kBatchRowLogMax; l >= 1; --l) {
        row32_by_size[l].insert(row32_by_size[l].end(), row32_tail[l].begin(), row32_tail[l].end());
        if (row32_by_size[l].empty()) continue;
        row_groups32_.push_back(RowGroup{l, int(items.size()), int(row32_by_size[l].size()), 0});
        items.insert(items.end(), row32_by_size[l].begin(), row32_by_size[l].end());
        shape.push_back((uint64_t(5) << 60) | (uint64_t(l) << 32) | uint64_t(row32_by_size[l].size()));
    }
    n_crt_tc32_ = int(crt_tc32.size());
    crt32_first_ = int(items.size());
    items.insert(items.end(), crt_tc32.begin(), crt_tc32.end());
    dec32_first_ = int(items.size());
    for (int l = 0; l <= kMaxLogN1; ++l) {
        n_dec_tc32_[l] = int(dec_tc32[l].size());
        items.insert(items.end(), dec_tc32[l].begin(), dec_tc32[l].end());
        shape.push_back((uint64_t(6) << 60) | (uint64_t(l) << 32) | uint64_t(n_dec_tc32_[l]));
    }
    shape.push_back((uint64_t(7) << 60) | (uint64_t(kmax32_) << 32) | (uint64_t(lw_tc32_) << 16) |
                    uint64_t(n_crt_tc32_));

    ensure(reinterpret_cast<char**>(&d_products_), &products_cap_, n * sizeof(BatchProduct), "batch products");
    ensure(&d_items_, &items_cap_, items.size(), "batch items");
    ensure(&d_state_, &state_cap_, 2 * n + 5 + 2 * kBatchRowLogMax, "batch counters");
    // Stream-ordered upload from pinned memory: the kernel on `stream` sees the tables only after
    // the copies (a synchronous copy from pageable memory may return before its DMA lands, and
    // nothing would order it before a launch on a non-blocking stream). The previous run has
    // completed (event above), so the pinned buffer is free to rewrite.
    const size_t prod_bytes = round_up(n * sizeof(BatchProduct), 256);
    const size_t item_bytes = items.size() * sizeof(uint2);
    if (prod_bytes + item_bytes > h_upload_cap_) {
        cudaFreeHost(h_upload_);
        h_upload_ = nullptr;
        h_upload_cap_ = 0;
        const size_t cap = 2 * (prod_bytes + item_bytes);
        check(cudaMallocHost(&h_upload_, cap), "batch upload staging");
        h_upload_cap_ = cap;
    }
    if (n) {
        std::memcpy(h_upload_, prods.data(), n * sizeof(BatchProduct));
        check(cudaMemcpyAsync(d_products_, h_upload_, n * sizeof(BatchProduct), cudaMemcpyHostToDevice, stream),
              "upload");
    }
    if (item_bytes) {
        std::memcpy(h_upload_ + prod_bytes, items.data(), item_bytes);
        check(cudaMemcpyAsync(d_items_, h_upload_ + prod_bytes, item_bytes, cudaMemcpyHostToDevice, stream), "upload");
    }

    smem_ = smax(kmax_imad > 0 ? dec_smem_bytes(kmax_imad) : 0, row_smem_bytes(kThreads, kBatchRowLogE));
    smem_dec_tc_ = dec_tc_smem_bytes(std::max(kmax_tc, 1));
    smem_crt_ = crt_smem_bytes(kmax);
    smem_crt_tc_ = crt_tc_smem_bytes(lw_tc);
    int per_sm = 0, sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "device attribute");
    if (with_dec_) {
        check(persistent_occupancy(smem_, &per_sm), "occupancy");
        ctas_ = std::max(1, std::min(per_sm * sms, n_items_));
    } else {
        ctas_ = 0;
        for (RowGroup& g : row_groups_) {
            check(persistent_rows_occupancy(g.logN2, &per_sm), "occupancy");
            g.ctas = std::max(1, std::min(per_sm * sms, g.count));
            ctas_ = std::max(ctas_, g.ctas);
        }
    }
    for (RowGroup& g : row_groups32_) {
        check(persistent_rows32_occupancy(g.logN2, &per_sm), "occupancy");
        g.ctas = std::max(1, std::min(per_sm * sms, g.count));
        ctas_ = std::max(ctas_, g.ctas);
    }
    if (shape != shape_) {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
        shape_ = shape;
    }
    dirty_ = false;
}

void Batch::run(cudaStream_t stream, bool use_graph) {
    if (entries_.empty()) return;
    if (dirty_) finalize(stream);
    const size_t n = entries_.size();
    BatchArgs args{};
    args.products = static_cast<const BatchProduct*>(d_products_);
    args.items = d_items_;
    args.n_items = n_items_;
    args.counters = d_state_;
    args.head = d_state_ + 2 * n;
    args.error = d_state_ + 2 * n + 1;
    args.tables = tables_->view();
    BatchCrtArgs tc{}, im{};
    tc.products = im.products = args.products;
    tc.tables = im.tables = args.tables;
    tc.items = d_items_ + n_items_;
    tc.n_items = n_crt_tc_;
    im.items = d_items_ + n_items_ + n_crt_tc_;
    im.n_items = n_crt_;
    // the tensor-core residue launches, the persistent launch, then the CRT launches (every row
    // item is done when they start)
    auto enqueue = [&](cudaStream_t s) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        if (!direct_.empty()) {
            // direct products alternate between s and the side stream (forked from s, joined below)
            e = cudaEventRecord(fork_, s);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(side_, fork_, 0);
            for (size_t j = 0; j < direct_.size() && e == cudaSuccess; ++j)
                e = launch_product(direct_[j].d, args.tables, direct_[j].cfg, (j & 1) ? side_ : s);
        }
        int at = n_items_ + n_crt_tc_ + n_crt_;
        for (int l = 0; l <= kMaxLogN1 && e == cudaSuccess; ++l) {
            if (n_dec_tc_[l] == 0) continue;
            BatchCrtArgs dt = tc;
            dt.items = d_items_ + at;
            dt.n_items = n_dec_tc_[l];
            e = launch_batch_dec_tc(dt, l, smem_dec_tc_, s);
            at += n_dec_tc_[l];
        }
        if (with_dec_) {
            if (e == cudaSuccess && n_items_ > 0) e = launch_persistent(args, ctas_, smem_, s);
        } else {
            for (size_t g = 0; g < row_groups_.size() && e == cudaSuccess; ++g) {
                BatchArgs ga = args;
                ga.items = d_items_ + row_groups_[g].first;
                ga.n_items = row_groups_[g].count;
                ga.head = d_state_ + 2 * n + 5 + g;
                e = launch_persistent_rows(ga, row_groups_[g].logN2, row_groups_[g].ctas, s);
            }
        }
        if (e == cudaSuccess && n_crt_tc_ > 0) e = launch_batch_crt(tc, true, smem_crt_tc_, s);
        if (e == cudaSuccess && n_crt_ > 0) e = launch_batch_crt(im, false, smem_crt_, s);
        // the 30-bit products: residue launches, persistent row launches, the CRT launch
        int at32 = dec32_first_;
        for (int l = 0; l <= kMaxLogN1 && e == cudaSuccess; ++l) {
            if (n_dec_tc32_[l] == 0) continue;
            BatchCrtArgs dt = tc;
            dt.items = d_items_ + at32;
            dt.n_items = n_dec_tc32_[l];
            e = launch_batch_dec_tc32(dt, l, kmax32_, s);
            at32 += n_dec_tc32_[l];
        }
        for (size_t g = 0; g < row_groups32_.size() && e == cudaSuccess; ++g) {
            BatchArgs ga = args;
            ga.items = d_items_ + row_groups32_[g].first;
            ga.n_items = row_groups32_[g].count;
            ga.head = d_state_ + 2 * n + 5 + kBatchRowLogMax + g;
            e = launch_persistent_rows32(ga, row_groups32_[g].logN2, row_groups32_[g].ctas, s);
        }
        if (e == cudaSuccess && n_crt_tc32_ > 0) {
            BatchCrtArgs ct = tc;
            ct.items = d_items_ + crt32_first_;
            ct.n_items = n_crt_tc32_;
            e = launch_batch_crt_tc32(ct, lw_tc32_, s);
        }
        if (!direct_.empty()) {
            // join the side stream back into s (also after a failed launch, so a capture ends whole)
            cudaError_t j = cudaEventRecord(join_, side_);
            if (j == cudaSuccess) j = cudaStreamWaitEvent(s, join_, 0);
            if (e == cudaSuccess) e = j;
        }
        return e;
    };
    const size_t state_bytes = (2 * n + 5 + 2 * kBatchRowLogMax) * sizeof(uint32_t);
    if (!use_graph) {
        check(cudaMemsetAsync(d_state_, 0, state_bytes, stream), "batch reset");
        check(enqueue(stream), "batch launch");
        check(cudaMemcpyAsync(err_host_, args.error, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), "batch status");
        check(cudaEventRecord(done_, stream), "batch event");
        ran_ = true;
        return;
    }
    if (!exec_) {
        cudaStream_t cap = nullptr;
        check(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaMemsetAsync(d_state_, 0, state_bytes, cap);
            const cudaError_t le = enqueue(cap);
            e = cudaStreamEndCapture(cap, &graph_);
            if (e == cudaSuccess) e = le;
        }
        cudaStreamDestroy(cap);
        check(e, "graph capture");
        check(cudaGraphInstantiate(&exec_, graph_, 0), "graph instantiate");
    }
    check(cudaGraphLaunch(exec_, stream), "graph launch");
    check(cudaMemcpyAsync(err_host_, args.error, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), "batch status");
    check(cudaEventRecord(done_, stream), "batch event");
    ran_ = true;
}

void Batch::synchronize() {
    if (!ran_) return;
    check(cudaEventSynchronize(done_), "batch");
    if (entries_.empty()) return;
    if (failed()) throw Error(kETimeout, failure());
}

std::string Batch::failure() const {
    if (!failed()) return std::string();
    return "a persistent-kernel dependency wait gave up (stage " + std::to_string(err_host_[1] >> 28) + ", product " +
           std::to_string(err_host_[1] & 0x0fffffffu) + ", saw " + std::to_string(err_host_[2]) + " of " +
           std::to_string(err_host_[3]) + ")";
}

}  // namespace nc
