// Exported entry points: the C ABI (negacyclic_b200.h) and the reference's C++ contract
// (fherma.h: fherma_init / fherma_run / fherma_free).
#include "fherma.h"
#include "negacyclic_b200.h"

#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"
#include "engine.h"
#include "hostmath.h"
#include "handles.h"
#include "kernel_registry.h"
#include "kernels.h"
#include "server.h"

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return NC_OK;
    } catch (const nc::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return NC_ENOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return NC_EINVAL;
    }
}

}  // namespace

void nc::set_last_error(const std::string& msg) { g_last_error = msg; }

extern "C" {

const char* nc_last_error(void) { return g_last_error.c_str(); }

int nc_version(void) { return 100; }

int nc_plan_create(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, nc_plan** out) {
    return guarded([&] {
        if (!out) throw nc::Error(nc::kEInval, "out is null");
        *out = nullptr;
        nc::Plan* p = nc::plan_create(N, W, L, q);
        *out = new nc_plan{p};
    });
}

int nc_self_check(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q) {
    return guarded([&] {
        if (N < 2 || N > uint32_t(nc::kMaxN) || (N & (N - 1)) != 0)
            throw nc::Error(nc::kEInval, "N must be a power of two from 2 to 65536");
        if (L == 0 || L > uint32_t(nc::kMaxL)) throw nc::Error(nc::kEInval, "L must be between 1 and 32");
        if (!q) throw nc::Error(nc::kEInval, "q is null");
        int logN = 0;
        while ((1u << logN) < N) ++logN;
        nc::QConst c{};
        const std::string err = nc::build_qconst(q, int(L), logN, &c);
        if (!err.empty()) throw nc::Error(nc::kEInval, err);
        if (W != 0 && (W < c.qbits || (W + 31) / 32 != L))
            throw nc::Error(nc::kEInval, "W must be the bit width of q and L = (W + 31) / 32");
        const std::string& host = nc::host_self_check();
        if (!host.empty()) throw nc::Error(nc::kESelfCheck, "init self-check: " + host);
        const std::string qerr = nc::check_qconst(c);
        if (!qerr.empty()) throw nc::Error(nc::kESelfCheck, "init self-check of the plan's constants: " + qerr);
        // the 30-bit engine's constants, where its 64 primes cover the bound
        nc::QConst32 c32{};
        if (nc::build_qconst32(q, int(L), logN, &c32).empty()) {
            const std::string e32 = nc::check_qconst32(c32);
            if (!e32.empty()) throw nc::Error(nc::kESelfCheck, "init self-check of the plan's 30-bit constants: " + e32);
        }
    });
}

int nc_plan_destroy(nc_plan* plan) {
    return guarded([&] {
        if (!plan) return;
        nc::plan_destroy(plan->p);
        delete plan;
    });
}

int nc_multiply(nc_plan* plan, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::plan_multiply_host(plan->p, a, b, c);
    });
}

int nc_multiply_device(nc_plan* plan, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, void* stream) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::plan_multiply_device(plan->p, d_a, d_b, d_c, static_cast<cudaStream_t>(stream));
    });
}

int nc_plan_create_chain(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int factors, nc_plan** out) {
    return guarded([&] {
        if (!out) throw nc::Error(nc::kEInval, "out is null");
        *out = nullptr;
        if (factors < 2 || factors > nc::kMaxFactors) throw nc::Error(nc::kEInval, "factors must be 2, 3 or 4");
        nc::Plan* p = nc::plan_create(N, W, L, q, factors);
        *out = new nc_plan{p};
    });
}

int nc_plan_factors(const nc_plan* plan) {
    if (!plan) {
        nc::set_last_error("null plan");
        return NC_EINVAL;
    }
    return plan->p->factors;
}

int nc_multiply_chain(nc_plan* plan, const uint32_t* const* x, uint32_t* c) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::plan_multiply_chain_host(plan->p, x, c);
    });
}

int nc_multiply_chain_device(nc_plan* plan, const uint32_t* const* d_x, uint32_t* d_c, void* stream) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::plan_multiply_chain_device(plan->p, d_x, d_c, static_cast<cudaStream_t>(stream));
    });
}

int nc_plan_set_crt_engine(nc_plan* plan, int engine) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        if (engine != NC_CRT_IMAD && engine != NC_CRT_TC_I8) throw nc::Error(nc::kEInval, "unknown CRT engine");
        if (engine == NC_CRT_TC_I8 && !plan->p->d_crt_b)
            throw nc::Error(nc::kEInval, "the tensor-core CRT takes at most 32 primes (q up to about 960 bits)");
        if (engine == NC_CRT_TC_I8 && !plan->p->tables->tensor_cores)
            throw nc::Error(nc::kEInval, "the tensor-core CRT needs a compute capability 10.0 device");
        plan->p->crt_tc = engine == NC_CRT_TC_I8;
    });
}

int nc_plan_get_crt_engine(const nc_plan* plan) {
    if (!plan) {
        nc::set_last_error("null plan");
        return NC_EINVAL;
    }
    return (plan->p->crt_tc && plan->p->d_crt_b) ? NC_CRT_TC_I8 : NC_CRT_IMAD;
}

int nc_plan_set_residue_engine(nc_plan* plan, int engine) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        if (engine != NC_RESIDUES_IMAD && engine != NC_RESIDUES_TC_I8) throw nc::Error(nc::kEInval, "unknown residue engine");
        if (engine == NC_RESIDUES_TC_I8 && !plan->p->tables->tensor_cores)
            throw nc::Error(nc::kEInval, "the tensor-core residue stage needs a compute capability 10.0 device");
        plan->p->res_tc = engine == NC_RESIDUES_TC_I8;
    });
}

int nc_plan_get_residue_engine(const nc_plan* plan) {
    if (!plan) {
        nc::set_last_error("null plan");
        return NC_EINVAL;
    }
    return plan->p->res_tc ? NC_RESIDUES_TC_I8 : NC_RESIDUES_IMAD;
}

int nc_plan_synchronize(nc_plan* plan) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::check(cudaStreamSynchronize(plan->p->stream), "synchronize");
    });
}

int nc_plan_query(const nc_plan* plan, uint32_t* N, uint32_t* L, uint32_t* k, uint32_t* qbits) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        if (N) *N = uint32_t(plan->p->N);
        if (L) *L = uint32_t(plan->p->L);
        if (k) *k = uint32_t(plan->p->k);
        if (qbits) *qbits = plan->p->hq.qbits;
    });
}

float nc_plan_last_kernel_ms(const nc_plan* plan) { return plan ? plan->p->last_kernel_ms : 0.f; }

int nc_plan_set_timing(nc_plan* plan, int enable) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        plan->p->timing = enable != 0;
    });
}

int nc_plan_stage_ms(const nc_plan* plan, float* ms) {
    return guarded([&] {
        if (!plan || !ms) throw nc::Error(nc::kEInval, "null argument");
        if (!plan->p->timing) throw nc::Error(nc::kEInval, "stage timing is off (nc_plan_set_timing)");
        for (int i = 0; i < 3; ++i)
            nc::check(cudaEventElapsedTime(&ms[i], plan->p->ev_stage[i], plan->p->ev_stage[i + 1]), "stage events");
    });
}

int nc_imad_peak(double* ops_per_second) {
    return guarded([&] {
        if (!ops_per_second) throw nc::Error(nc::kEInval, "null argument");
        nc::check(nc::measure_imad_peak(ops_per_second), "IMAD probe");
    });
}

int nc_primes(uint64_t* out, int count) {
    return guarded([&] {
        if (!out || count < 0 || count > nc::kMaxPrimes) throw nc::Error(nc::kEInval, "count must be 0..48");
        const auto& ps = nc::prime_set();
        for (int i = 0; i < count; ++i) out[i] = ps[i].p;
    });
}

int nc_primes32(uint32_t* out, int count) {
    return guarded([&] {
        if (!out || count < 0 || count > nc::kMaxPrimes32) throw nc::Error(nc::kEInval, "count must be 0..64");
        const auto& ps = nc::prime_set32();
        for (int i = 0; i < count; ++i) out[i] = ps[size_t(i)].p;
    });
}

}  // extern "C"

// ------------------------------------------------------------------ reference contract

namespace {

// The state behind the contract's void*: the plan, plus the next call's output vector. A
// std::vector<uint32_t> of N*L elements must be value-initialised before it has that size, a
// 7 MB memset at N = 65536; a helper thread prepares the next one after each call returns, so
// fherma_run only moves a ready vector into its Outputs.
struct FhermaState {
    nc::Plan* plan = nullptr;
    std::vector<uint32_t> spare;
    std::mutex mu;
    std::condition_variable cv;
    bool want = false, stop = false;
    std::thread helper;

    explicit FhermaState(nc::Plan* p) : plan(p), spare(p->limbs()) {
        helper = std::thread([this] {
            std::unique_lock<std::mutex> lock(mu);
            for (;;) {
                cv.wait(lock, [&] { return want || stop; });
                if (stop) return;
                lock.unlock();
                std::vector<uint32_t> v(plan->limbs());
                lock.lock();
                spare = std::move(v);
                want = false;
                cv.notify_all();
            }
        });
    }
    ~FhermaState() {
        {
            std::lock_guard<std::mutex> lock(mu);
            stop = true;
        }
        cv.notify_all();
        helper.join();
        nc::plan_destroy(plan);
    }
    std::vector<uint32_t> take() {
        std::unique_lock<std::mutex> lock(mu);
        cv.wait(lock, [&] { return !want; });
        std::vector<uint32_t> v = std::move(spare);
        want = true;  // the helper builds the next one while the caller uses this one
        cv.notify_all();
        return v;
    }
};

}  // namespace

void* fherma_init(const fherma::Point& point) {
    if (point.q.data.size() != point.L) throw std::runtime_error("q must hold L limbs");
    try {
        nc::Plan* p = nc::plan_create(point.N, point.W, point.L, point.q.data.data());
        try {
            // init is not timed by the harness: pick the row tiling for this N on the device now
            const char* tune = std::getenv("NC_AUTOTUNE");
            if (!(tune && tune[0] == '0')) nc::plan_autotune(p, 3);
            nc::ensure_host_path(p);
            return new FhermaState(p);
        } catch (...) {
            nc::plan_destroy(p);
            throw;
        }
    } catch (const nc::Error& e) {
        throw std::runtime_error(e.what());
    }
}

fherma::Outputs fherma_run(void* state, const fherma::Inputs& in) {
    auto* st = static_cast<FhermaState*>(state);
    if (!st) throw std::runtime_error("null state");
    nc::Plan* p = st->plan;
    const size_t count = p->limbs();
    if (in.a.data.size() != count || in.b.data.size() != count)
        throw std::runtime_error("a and b must contain N*L limbs");
    fherma::Outputs out;
    out.c.shape = {int64_t(p->N), int64_t(p->L)};
    try {
        nc::plan_submit_host(p, in.a.data.data(), in.b.data.data());
        out.c.data = st->take();
        if (out.c.data.size() != count) out.c.data.resize(count);
        nc::plan_collect_host(p, out.c.data.data());
    } catch (const nc::Error& e) {
        throw std::runtime_error(e.what());
    }
    return out;
}

void fherma_free(void* state) { delete static_cast<FhermaState*>(state); }

// ------------------------------------------------------------------ tuning and batches

struct nc_batch {
    nc::Batch* b;
};

extern "C" {

int nc_row_variants(uint32_t log_n, int* triples, int max_variants) {
    if (log_n < 1 || log_n > uint32_t(nc::kMaxLogN) || (!triples && max_variants > 0)) {
        g_last_error = "log_n must be 1..16";
        return NC_EINVAL;
    }
    const auto v = nc::row_variants(int(log_n));
    int n = 0;
    for (const auto& c : v) {
        if (n >= max_variants) break;
        triples[3 * n] = c.logN2;
        triples[3 * n + 1] = c.logE;
        triples[3 * n + 2] = c.threads;
        ++n;
    }
    return max_variants <= 0 ? int(v.size()) : n;
}

int nc_plan_set_row_config(nc_plan* plan, int log_block, int log_radix, int threads) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::plan_set_row_config(plan->p, nc::RowConfig{log_block, log_radix, threads});
    });
}

int nc_plan_get_row_config(const nc_plan* plan, int* log_block, int* log_radix, int* threads) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        const nc::RowConfig& c = plan->p->plain_cfg();
        if (log_block) *log_block = c.logN2;
        if (log_radix) *log_radix = c.logE;
        if (threads) *threads = c.threads;
    });
}

int nc_row_variants32(uint32_t log_n, int* triples, int max_variants) {
    if (log_n < 1 || log_n > uint32_t(nc::kMaxLogN) || (!triples && max_variants > 0)) {
        g_last_error = "log_n must be 1..16";
        return NC_EINVAL;
    }
    std::vector<nc::RowConfig> v;
    for (const nc::RowConfig& c : nc::all_row32_variants())
        if (nc::row_config_valid(int(log_n), c)) v.push_back(c);
    int n = 0;
    for (const auto& c : v) {
        if (n >= max_variants) break;
        triples[3 * n] = c.logN2;
        triples[3 * n + 1] = c.logE;
        triples[3 * n + 2] = c.threads;
        ++n;
    }
    return max_variants <= 0 ? int(v.size()) : n;
}

int nc_plan_set_word_bits(nc_plan* plan, int bits) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        nc::plan_set_word_bits(plan->p, bits);
    });
}

int nc_plan_word_bits(const nc_plan* plan, uint32_t* k) {
    if (!plan) {
        g_last_error = "null plan";
        return NC_EINVAL;
    }
    const bool w32 = plan->p->use_w32();
    if (k) *k = uint32_t(w32 ? plan->p->k32 : plan->p->k);
    return w32 ? 32 : 64;
}

int nc_plan_autotune(nc_plan* plan, int reps, float* best_ms) {
    return guarded([&] {
        if (!plan) throw nc::Error(nc::kEInval, "null plan");
        const float ms = nc::plan_autotune(plan->p, reps);
        if (best_ms) *best_ms = ms;
    });
}

uint64_t nc_plan_hat_words(const nc_plan* plan) {
    // k N u64 words on the 62-bit engine; k32 N u32 values on the 30-bit one (the larger of the two)
    return plan ? uint64_t((plan->p->residue_bytes() + 7) / 8) : 0;
}

int nc_batch_create(nc_batch** out) {
    return guarded([&] {
        if (!out) throw nc::Error(nc::kEInval, "out is null");
        *out = nullptr;
        auto* b = new nc::Batch(nc::current_device());
        *out = new nc_batch{b};
    });
}

int nc_batch_destroy(nc_batch* batch) {
    return guarded([&] {
        if (!batch) return;
        delete batch->b;
        delete batch;
    });
}

int nc_batch_add(nc_batch* batch, nc_plan* plan, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c) {
    return guarded([&] {
        if (!batch || !plan) throw nc::Error(nc::kEInval, "null batch or plan");
        batch->b->add(plan->p, nc::kModeProduct, d_a, d_b, d_c, nullptr, nullptr);
    });
}

int nc_batch_add_cached(nc_batch* batch, nc_plan* plan, const uint64_t* d_a_hat, const uint32_t* d_b, uint32_t* d_c) {
    return guarded([&] {
        if (!batch || !plan) throw nc::Error(nc::kEInval, "null batch or plan");
        batch->b->add(plan->p, nc::kModeCachedA, nullptr, d_b, d_c, d_a_hat, nullptr);
    });
}

int nc_batch_add_forward(nc_batch* batch, nc_plan* plan, const uint32_t* d_a, uint64_t* d_a_hat) {
    return guarded([&] {
        if (!batch || !plan) throw nc::Error(nc::kEInval, "null batch or plan");
        batch->b->add(plan->p, nc::kModeForward, d_a, nullptr, nullptr, nullptr, d_a_hat);
    });
}

int nc_batch_clear(nc_batch* batch) {
    return guarded([&] {
        if (!batch) throw nc::Error(nc::kEInval, "null batch");
        batch->b->clear();
    });
}

int nc_batch_run(nc_batch* batch, void* stream, int use_graph) {
    return guarded([&] {
        if (!batch) throw nc::Error(nc::kEInval, "null batch");
        batch->b->run(static_cast<cudaStream_t>(stream), use_graph != 0);
    });
}

int nc_batch_synchronize(nc_batch* batch) {
    return guarded([&] {
        if (!batch) throw nc::Error(nc::kEInval, "null batch");
        batch->b->synchronize();
    });
}

int nc_batch_query(const nc_batch* batch, uint32_t* products, uint32_t* ctas, uint64_t* scratch_bytes) {
    return guarded([&] {
        if (!batch) throw nc::Error(nc::kEInval, "null batch");
        if (products) *products = uint32_t(batch->b->size());
        if (ctas) *ctas = uint32_t(batch->b->ctas());
        if (scratch_bytes) *scratch_bytes = uint64_t(batch->b->scratch_bytes());
    });
}

}  // extern "C"

// ------------------------------------------------------------------ serving

struct nc_server {
    nc::Server* s;
};

extern "C" {

int nc_server_create(uint64_t hbm_budget_bytes, uint64_t staging_bytes, int max_batch, int streams, nc_server** out) {
    return guarded([&] {
        if (!out) throw nc::Error(nc::kEInval, "out is null");
        *out = nullptr;
        auto* s = new nc::Server(nc::current_device(), size_t(hbm_budget_bytes), size_t(staging_bytes), max_batch,
                                 streams);
        *out = new nc_server{s};
    });
}

int nc_server_destroy(nc_server* server) {
    return guarded([&] {
        if (!server) return;
        delete server->s;
        delete server;
    });
}

int nc_server_register_operand(nc_server* server, nc_plan* plan, const uint32_t* a, int* operand_id) {
    return guarded([&] {
        if (!server || !plan || !operand_id) throw nc::Error(nc::kEInval, "null argument");
        *operand_id = server->s->register_operand(plan->p, a);
    });
}

int nc_server_release_operand(nc_server* server, int operand_id) {
    return guarded([&] {
        if (!server) throw nc::Error(nc::kEInval, "null server");
        server->s->release_operand(operand_id);
    });
}

int nc_server_submit(nc_server* server, nc_plan* plan, const uint32_t* a, int operand_id, const uint32_t* b,
                     uint64_t* request_id) {
    return guarded([&] {
        if (!server || !plan || !request_id) throw nc::Error(nc::kEInval, "null argument");
        *request_id = server->s->submit(plan->p, a, operand_id, b);
    });
}

int nc_server_poll(nc_server* server, uint64_t request_id) {
    int r = 0;
    const int st = guarded([&] {
        if (!server) throw nc::Error(nc::kEInval, "null server");
        r = server->s->done(request_id) ? 1 : 0;
    });
    return st == NC_OK ? r : st;
}

int nc_server_wait(nc_server* server, uint64_t request_id, uint32_t* c, double* latency_ms) {
    return guarded([&] {
        if (!server) throw nc::Error(nc::kEInval, "null server");
        const double ms = server->s->wait(request_id, c);
        if (latency_ms) *latency_ms = ms;
    });
}

int nc_server_stats(nc_server* server, double* p50_ms, double* p99_ms, uint64_t* completed, double* products_per_s,
                    uint64_t* hbm_in_use, uint64_t* batches, uint64_t* timeouts) {
    return guarded([&] {
        if (!server) throw nc::Error(nc::kEInval, "null server");
        size_t in_use = 0;
        uint64_t done = 0, b = 0, t = 0;
        server->s->stats(p50_ms, p99_ms, &done, products_per_s, &in_use, &b, &t);
        if (completed) *completed = done;
        if (hbm_in_use) *hbm_in_use = in_use;
        if (batches) *batches = b;
        if (timeouts) *timeouts = t;
    });
}

int nc_server_io_stats(nc_server* server, uint64_t* h2d_bytes, uint64_t* d2h_bytes, double* device_busy_ms,
                       double* device_window_ms, double* scheduler_ms) {
    return guarded([&] {
        if (!server) throw nc::Error(nc::kEInval, "null server");
        server->s->io_stats(h2d_bytes, d2h_bytes, device_busy_ms, device_window_ms, scheduler_ms);
    });
}

}  // extern "C"
