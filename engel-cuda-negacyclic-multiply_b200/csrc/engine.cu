// Plans, device tables and the host-buffer pipeline (see engine.h).
#include "engine.h"

#include <cstdlib>
#include <cstring>
#include <map>

#include "hostmath.h"
#include "kernels.h"

namespace nc {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? kENoMem : kECuda;
        throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

int current_device() {
    int d = 0;
    check(cudaGetDevice(&d), "cudaGetDevice");
    return d;
}

// ------------------------------------------------------------------------------ tables

namespace {
std::mutex g_tables_mu;
std::map<int, DeviceTables*> g_tables;
}  // namespace

DeviceTables* acquire_tables(int device) {
    std::lock_guard<std::mutex> lock(g_tables_mu);
    auto it = g_tables.find(device);
    if (it != g_tables.end()) {
        ++it->second->refs;
        return it->second;
    }
    const HostTables& h = host_tables();
    for (const auto& c : h.pc)
        if (c.m >= (1ull << 28)) throw Error(kEInval, "internal: prime set outside the 2^62 - m, m < 2^28 shape");
    auto* t = new DeviceTables();
    t->device = device;
    try {
        const size_t tw_bytes = size_t(kMaxPrimes) * kMaxN * sizeof(ulonglong2);
        check(cudaMalloc(&t->fwd, tw_bytes), "twiddle table");
        check(cudaMalloc(&t->inv, tw_bytes), "inverse twiddle table");
        check(cudaMalloc(&t->pow32, h.pow32.size() * sizeof(uint64_t)), "residue places");
        check(cudaMalloc(&t->pc, h.pc.size() * sizeof(PrimeConst)), "prime constants");
        check(cudaMemcpy(t->fwd, h.fwd.data(), tw_bytes, cudaMemcpyHostToDevice), "twiddle upload");
        check(cudaMemcpy(t->inv, h.inv.data(), tw_bytes, cudaMemcpyHostToDevice), "inverse twiddle upload");
        check(cudaMemcpy(t->pow32, h.pow32.data(), h.pow32.size() * sizeof(uint64_t), cudaMemcpyHostToDevice),
              "residue places upload");
        check(cudaMemcpy(t->pc, h.pc.data(), h.pc.size() * sizeof(PrimeConst), cudaMemcpyHostToDevice),
              "prime constants upload");
        check(prepare_plain_kernels(), "kernel attributes");
    } catch (...) {
        cudaFree(t->fwd);
        cudaFree(t->inv);
        cudaFree(t->pow32);
        cudaFree(t->pc);
        delete t;
        throw;
    }
    t->refs = 1;
    g_tables[device] = t;
    return t;
}

void release_tables(DeviceTables* t) {
    if (!t) return;
    std::lock_guard<std::mutex> lock(g_tables_mu);
    if (--t->refs > 0) return;
    g_tables.erase(t->device);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(t->device);
    cudaFree(t->fwd);
    cudaFree(t->inv);
    cudaFree(t->pow32);
    cudaFree(t->pc);
    cudaSetDevice(prev);
    delete t;
}

// ------------------------------------------------------------------------------ host copies

ParallelCopy::ParallelCopy(int threads) {
    for (int w = 1; w < threads; ++w)
        workers_.emplace_back([this, w] {
            uint64_t seen = 0;
            for (;;) {
                {
                    std::unique_lock<std::mutex> lock(mu_);
                    cv_.wait(lock, [&] { return stop_ || gen_ != seen; });
                    if (stop_) return;
                    seen = gen_;
                }
                run_part(w);
                std::lock_guard<std::mutex> lock(mu_);
                if (--pending_ == 0) done_cv_.notify_all();
            }
        });
}

ParallelCopy::~ParallelCopy() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
}

void ParallelCopy::run_part(int part) {
    const size_t parts = workers_.size() + 1;
    const size_t chunk = ((bytes_ + parts - 1) / parts + 63) & ~size_t(63);
    const size_t begin = chunk * size_t(part);
    if (begin >= bytes_) return;
    const size_t n = (begin + chunk > bytes_) ? bytes_ - begin : chunk;
    std::memcpy(dst_ + begin, src_ + begin, n);
}

void ParallelCopy::copy(void* dst, const void* src, size_t bytes) {
    if (workers_.empty() || bytes < (size_t(1) << 20)) {
        std::memcpy(dst, src, bytes);
        return;
    }
    {
        std::lock_guard<std::mutex> lock(mu_);
        dst_ = static_cast<char*>(dst);
        src_ = static_cast<const char*>(src);
        bytes_ = bytes;
        pending_ = int(workers_.size());
        ++gen_;
    }
    cv_.notify_all();
    run_part(0);
    std::unique_lock<std::mutex> lock(mu_);
    done_cv_.wait(lock, [&] { return pending_ == 0; });
}

// ------------------------------------------------------------------------------ plans

ProductDesc Plan::desc(const uint32_t* a, const uint32_t* b, uint32_t* c) const {
    ProductDesc d{};
    d.a = a;
    d.b = b;
    d.c = c;
    d.ra = d_ra;
    d.rb = d_rb;
    d.qc = d_qc;
    d.logN = uint32_t(logN);
    d.L = uint32_t(L);
    d.LW = hq.LW;
    d.k = uint32_t(k);
    d.mode = kModeProduct;
    return d;
}

static int copy_threads() {
    if (const char* s = std::getenv("NC_COPY_THREADS")) {
        const int v = std::atoi(s);
        if (v >= 1 && v <= 64) return v;
    }
    const int hc = int(std::thread::hardware_concurrency());
    return hc < 2 ? 1 : (hc < 8 ? hc : 8);
}

Plan* plan_create(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q) {
    if (N < 2 || N > uint32_t(kMaxN) || (N & (N - 1)) != 0)
        throw Error(kEInval, "N must be a power of two from 2 to 65536");
    if (L == 0 || L > uint32_t(kMaxL)) throw Error(kEInval, "L must be between 1 and 32");
    if (q == nullptr) throw Error(kEInval, "q is null");
    int logN = 0;
    while ((1u << logN) < N) ++logN;
    auto* p = new Plan();
    p->N = int(N);
    p->L = int(L);
    p->logN = logN;
    const std::string err = build_qconst(q, int(L), logN, &p->hq);
    if (!err.empty()) {
        delete p;
        throw Error(kEInval, err);
    }
    p->W = W ? int(W) : int(p->hq.qbits);
    if (W != 0 && (W < p->hq.qbits || (W + 31) / 32 != L)) {
        delete p;
        throw Error(kEInval, "W must be the bit width of q and L = (W + 31) / 32");
    }
    p->k = int(p->hq.k);
    try {
        p->device = current_device();
        p->tables = acquire_tables(p->device);
        const size_t res = size_t(p->k) * N * sizeof(uint64_t);
        const size_t limbs = size_t(N) * L * sizeof(uint32_t);
        check(cudaMalloc(&p->d_qc, sizeof(QConst)), "plan constants");
        check(cudaMemcpy(p->d_qc, &p->hq, sizeof(QConst), cudaMemcpyHostToDevice), "plan constants upload");
        check(cudaMalloc(&p->d_ra, res), "residues a");
        check(cudaMalloc(&p->d_rb, res), "residues b");
        check(cudaMalloc(&p->d_a, limbs), "input a");
        check(cudaMalloc(&p->d_b, limbs), "input b");
        check(cudaMalloc(&p->d_c, limbs), "output c");
        check(cudaMallocHost(&p->h_a, limbs), "pinned a");
        check(cudaMallocHost(&p->h_b, limbs), "pinned b");
        check(cudaMallocHost(&p->h_c, limbs), "pinned c");
        check(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "stream");
        check(cudaEventCreate(&p->ev_start), "event");
        check(cudaEventCreate(&p->ev_stop), "event");
        for (auto& ev : p->ev_stage) check(cudaEventCreate(&ev), "event");
        p->copier = new ParallelCopy(copy_threads());
    } catch (...) {
        plan_destroy(p);
        throw;
    }
    return p;
}

void plan_destroy(Plan* p) {
    if (!p) return;
    if (p->stream) cudaStreamSynchronize(p->stream);
    cudaFree(p->d_qc);
    cudaFree(p->d_ra);
    cudaFree(p->d_rb);
    cudaFree(p->d_a);
    cudaFree(p->d_b);
    cudaFree(p->d_c);
    cudaFreeHost(p->h_a);
    cudaFreeHost(p->h_b);
    cudaFreeHost(p->h_c);
    if (p->ev_start) cudaEventDestroy(p->ev_start);
    if (p->ev_stop) cudaEventDestroy(p->ev_stop);
    for (auto ev : p->ev_stage)
        if (ev) cudaEventDestroy(ev);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p->copier;
    release_tables(p->tables);
    delete p;
}

void plan_multiply_device(Plan* p, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t stream) {
    if (!p) throw Error(kEInval, "null plan");
    if (!d_a || !d_b || !d_c) throw Error(kEInval, "null device buffer");
    if (((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_b) | reinterpret_cast<uintptr_t>(d_c)) &
         15) != 0)
        throw Error(kEInval, "device buffers must be 16-byte aligned");
    const ProductDesc d = p->desc(d_a, d_b, d_c);
    check(launch_product(d, p->tables->view(), stream, p->timing ? p->ev_stage : nullptr), "kernel launch");
}

void plan_multiply_host(Plan* p, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (!p) throw Error(kEInval, "null plan");
    if (!a || !b || !c) throw Error(kEInval, "null host buffer");
    const size_t bytes = p->limbs() * sizeof(uint32_t);
    p->copier->copy(p->h_a, a, bytes);
    check(cudaMemcpyAsync(p->d_a, p->h_a, bytes, cudaMemcpyHostToDevice, p->stream), "a copy");
    p->copier->copy(p->h_b, b, bytes);
    check(cudaMemcpyAsync(p->d_b, p->h_b, bytes, cudaMemcpyHostToDevice, p->stream), "b copy");
    check(cudaEventRecord(p->ev_start, p->stream), "event");
    check(launch_product(p->desc(p->d_a, p->d_b, p->d_c), p->tables->view(), p->stream,
                         p->timing ? p->ev_stage : nullptr),
          "kernel launch");
    check(cudaEventRecord(p->ev_stop, p->stream), "event");
    check(cudaMemcpyAsync(p->h_c, p->d_c, bytes, cudaMemcpyDeviceToHost, p->stream), "c copy");
    check(cudaStreamSynchronize(p->stream), "product");
    cudaEventElapsedTime(&p->last_kernel_ms, p->ev_start, p->ev_stop);
    p->copier->copy(c, p->h_c, bytes);
}

}  // namespace nc
