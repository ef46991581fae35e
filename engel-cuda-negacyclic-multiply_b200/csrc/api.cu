// Exported entry points: the C ABI (negacyclic_b200.h) and the reference's C++ contract
// (fherma.h: fherma_init / fherma_run / fherma_free).
#include "fherma.h"
#include "negacyclic_b200.h"

#include <cstring>
#include <string>

#include "engine.h"
#include "hostmath.h"
#include "kernels.h"

struct nc_plan {
    nc::Plan* p;
};

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

}  // extern "C"

// ------------------------------------------------------------------ reference contract

void* fherma_init(const fherma::Point& point) {
    if (point.q.data.size() != point.L) throw std::runtime_error("q must hold L limbs");
    try {
        return nc::plan_create(point.N, point.W, point.L, point.q.data.data());
    } catch (const nc::Error& e) {
        throw std::runtime_error(e.what());
    }
}

fherma::Outputs fherma_run(void* state, const fherma::Inputs& in) {
    auto* p = static_cast<nc::Plan*>(state);
    if (!p) throw std::runtime_error("null state");
    const size_t count = p->limbs();
    if (in.a.data.size() != count || in.b.data.size() != count)
        throw std::runtime_error("a and b must contain N*L limbs");
    fherma::Outputs out;
    out.c.shape = {int64_t(p->N), int64_t(p->L)};
    out.c.data.resize(count);
    try {
        nc::plan_multiply_host(p, in.a.data.data(), in.b.data.data(), out.c.data.data());
    } catch (const nc::Error& e) {
        throw std::runtime_error(e.what());
    }
    return out;
}

void fherma_free(void* state) { nc::plan_destroy(static_cast<nc::Plan*>(state)); }
