// Plans, device tables and the host-buffer pipeline (see engine.h).
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

#include "hostcopy.h"
#include "hostmath.h"
#include "kernel_registry.h"
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

void free_tables(DeviceTables* t) {
    for (void* ptr : {static_cast<void*>(t->fwd), static_cast<void*>(t->inv), static_cast<void*>(t->pow32),
                      static_cast<void*>(t->primes), static_cast<void*>(t->res_w), static_cast<void*>(t->fwd32),
                      static_cast<void*>(t->inv32), static_cast<void*>(t->pc32), static_cast<void*>(t->pow32_32),
                      static_cast<void*>(t->res_w32)})
        cudaFree(ptr);
}

// The 30-bit engine's tables: twiddles (w, floor(w 2^32 / p)), prime constants, 2^(32 l) mod p,
// and the residue stage's weight bytes (byte c of 2^(8 b) mod p_i at
// [i / 2][b / 16][4 (i % 2) + c][b % 16], b < 128: the MMA's B rows of a prime pair).
void upload_tables32(DeviceTables* t) {
    const HostTables32& h = host_tables32();
    const size_t tw = size_t(kMaxPrimes32) * kMaxN * sizeof(uint2);
    check(cudaMalloc(&t->fwd32, tw), "30-bit twiddle table");
    check(cudaMalloc(&t->inv32, tw), "30-bit inverse twiddle table");
    check(cudaMemcpy(t->fwd32, h.fwd.data(), tw, cudaMemcpyHostToDevice), "30-bit twiddle upload");
    check(cudaMemcpy(t->inv32, h.inv.data(), tw, cudaMemcpyHostToDevice), "30-bit inverse twiddle upload");
    check(cudaMalloc(&t->pc32, size_t(kMaxPrimes32) * sizeof(PrimeConst32)), "30-bit prime table");
    check(cudaMemcpy(t->pc32, h.pc.data(), size_t(kMaxPrimes32) * sizeof(PrimeConst32), cudaMemcpyHostToDevice),
          "30-bit prime upload");
    check(cudaMalloc(&t->pow32_32, size_t(kMaxPrimes32) * kMaxL * 4), "30-bit limb weights");
    check(cudaMemcpy(t->pow32_32, h.pow32.data(), size_t(kMaxPrimes32) * kMaxL * 4, cudaMemcpyHostToDevice),
          "30-bit limb weight upload");
    std::vector<uint8_t> w(size_t(kMaxPrimes32 / 2) * 1024, 0);
    for (int i = 0; i < kMaxPrimes32; ++i) {
        const uint64_t p = h.pc[size_t(i)].p;
        uint64_t v = 1;
        for (int b = 0; b < 128; ++b) {
            for (int c = 0; c < 4; ++c)
                w[size_t(i / 2) * 1024 + size_t(b / 16) * 128 + size_t(4 * (i % 2) + c) * 16 + size_t(b % 16)] =
                    uint8_t(v >> (8 * c));
            v = v * 256u % p;
        }
    }
    check(cudaMalloc(&t->res_w32, w.size()), "30-bit residue weight table");
    check(cudaMemcpy(t->res_w32, w.data(), w.size(), cudaMemcpyHostToDevice), "30-bit residue weight upload");
}
}  // namespace

DeviceTables* acquire_tables(int device) {
    std::lock_guard<std::mutex> lock(g_tables_mu);
    auto it = g_tables.find(device);
    if (it != g_tables.end()) {
        ++it->second->refs;
        return it->second;
    }
    const HostTables& h = host_tables();
    const std::string& host_err = host_self_check();
    if (!host_err.empty()) throw Error(kESelfCheck, "init self-check: " + host_err);
    auto* t = new DeviceTables();
    t->device = device;
    try {
        int major = 0, minor = 0;
        check(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "device attribute");
        check(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device), "device attribute");
        t->tensor_cores = NC_HAS_TCGEN05 && major == 10 && minor == 0;
        const size_t tw_bytes = size_t(kMaxPrimes) * kMaxN * sizeof(ulonglong2);
        check(cudaMalloc(&t->fwd, tw_bytes), "twiddle table");
        check(cudaMalloc(&t->inv, tw_bytes), "inverse twiddle table");
        check(cudaMemcpy(t->fwd, h.fwd.data(), tw_bytes, cudaMemcpyHostToDevice), "twiddle upload");
        check(cudaMemcpy(t->inv, h.inv.data(), tw_bytes, cudaMemcpyHostToDevice), "inverse twiddle upload");
        std::vector<uint64_t> primes(kMaxPrimes);
        for (int i = 0; i < kMaxPrimes; ++i) primes[size_t(i)] = h.pc[size_t(i)].p;
        check(cudaMalloc(&t->pow32, size_t(kMaxPrimes) * kMaxL * sizeof(uint64_t)), "limb weights");
        check(cudaMalloc(&t->primes, size_t(kMaxPrimes) * sizeof(uint64_t)), "prime table");
        check(cudaMemcpy(t->pow32, h.pow32.data(), size_t(kMaxPrimes) * kMaxL * sizeof(uint64_t),
                         cudaMemcpyHostToDevice),
              "limb weight upload");
        check(cudaMemcpy(t->primes, primes.data(), size_t(kMaxPrimes) * sizeof(uint64_t), cudaMemcpyHostToDevice),
              "prime upload");
        // weight bytes of the tensor-core residue stage: byte c of 2^(8 b) mod p_i at
        // [i][b / 16][c][b % 16], b < 128 (the K bytes of up to 32 limbs)
        std::vector<uint8_t> w(size_t(kMaxPrimes) * 1024, 0);
        for (int i = 0; i < kMaxPrimes; ++i) {
            const uint64_t p = h.pc[size_t(i)].p;
            uint64_t v = 1;
            for (int b = 0; b < 128; ++b) {
                for (int c = 0; c < 8; ++c)
                    w[size_t(i) * 1024 + size_t(b / 16) * 128 + size_t(c) * 16 + size_t(b % 16)] = uint8_t(v >> (8 * c));
                v = uint64_t((unsigned __int128)v * 256u % p);
            }
        }
        check(cudaMalloc(&t->res_w, w.size()), "residue weight table");
        check(cudaMemcpy(t->res_w, w.data(), w.size(), cudaMemcpyHostToDevice), "residue weight upload");
        if (t->tensor_cores) upload_tables32(t);
        check(prepare_kernels(h.pc.data(), h.pow32.data()), "kernel preparation");
        check(prepare_noalloc(device), "allocation-free scratch set-up");
        // a synchronous copy from pageable memory may return before its last DMA lands, and the
        // kernels run on non-blocking streams that do not order after it: wait for the device
        check(cudaDeviceSynchronize(), "table upload");
    } catch (...) {
        free_tables(t);
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
    free_tables(t);
    cudaSetDevice(prev);
    delete t;
}

// Host-side self-checks, once per process: known answers of the host arithmetic, both prime
// sets, and a sample of every prime's tables (psi, 2^(32 l) mod p, twiddles and Shoup companions).
const std::string& host_self_check() {
    static std::string err;
    static std::once_flag once;
    std::call_once(once, [] {
        err = check_arithmetic();
        if (err.empty()) err = check_prime_set();
        if (err.empty()) err = check_tables(host_tables(), 64);
        if (err.empty()) err = check_prime_set32();
        if (err.empty()) err = check_tables32(host_tables32(), 64);
    });
    return err;
}

// ------------------------------------------------------------------------------ host pool

HostPool::HostPool(int threads) {
    for (int w = 1; w < threads; ++w) workers_.emplace_back([this, w] { worker(w); });
}

HostPool::~HostPool() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        stop_.store(true);
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
}

void HostPool::worker(int part) {
    uint64_t seen = 0;
    for (;;) {
        // spin for a short while (jobs of one product come back to back), then sleep
        const auto spin_until = std::chrono::steady_clock::now() + std::chrono::microseconds(300);
        while (gen_.load(std::memory_order_acquire) == seen && !stop_.load() &&
               std::chrono::steady_clock::now() < spin_until) {
        }
        if (gen_.load(std::memory_order_acquire) == seen && !stop_.load()) {
            std::unique_lock<std::mutex> lock(mu_);
            cv_.wait(lock, [&] { return stop_.load() || gen_.load() != seen; });
        }
        if (stop_.load()) return;
        seen = gen_.load(std::memory_order_acquire);
        (*job_)(part, parts());
        pending_.fetch_sub(1, std::memory_order_acq_rel);
    }
}

void HostPool::run(const std::function<void(int, int)>& fn) {
    if (workers_.empty()) {
        fn(0, 1);
        return;
    }
    std::lock_guard<std::mutex> one_job(run_mu_);  // callers on several threads take turns
    job_ = &fn;
    pending_.store(int(workers_.size()), std::memory_order_relaxed);
    {
        std::lock_guard<std::mutex> lock(mu_);
        gen_.fetch_add(1, std::memory_order_acq_rel);
    }
    cv_.notify_all();
    fn(0, parts());
    while (pending_.load(std::memory_order_acquire) != 0) {
    }
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
    d.logN2 = uint32_t(cfg.logN2);
    d.crt_b = crt_tc ? d_crt_b : nullptr;
    d.factors = 2;
    d.res_tc = res_tc ? 1u : 0u;
    return d;
}

ProductDesc Plan::desc_plain(const uint32_t* a, const uint32_t* b, uint32_t* c) const {
    ProductDesc d = desc(a, b, c);
    if (use_w32()) {
        d.k = uint32_t(k32);
        d.qc32 = d_qc32;
        d.crt_b = d_crt_b32;
        d.logN2 = uint32_t(cfg32.logN2);
        d.res_tc = 1u;
    }
    return d;
}

size_t Plan::residue_bytes() const {
    const size_t r64 = size_t(k) * size_t(N) * sizeof(uint64_t);
    const size_t r32 = size_t(k32) * size_t(N) * sizeof(uint32_t);
    return r64 > r32 ? r64 : r32;
}

ProductDesc Plan::desc_chain(const uint32_t* const* x, uint32_t* c) const {
    ProductDesc d = desc(x[0], x[1], c);
    d.factors = uint32_t(factors);
    for (int f = 2; f < factors; ++f) {
        d.x_more[f - 2] = x[f];
        d.r_more[f - 2] = d_rx[f - 2];
    }
    return d;
}

namespace {

// Table B of the tensor-core CRT in the MMA's shared-memory order: output byte column c, K byte
// 8 i + a holds byte c - a of (M/p_i) mod q (zero outside 0 <= c - a < 4 L), stored at
// (c / 8) * 2048 + (K / 16) * 128 + (c % 8) * 16 + K % 16.
std::vector<uint8_t> crt_tc_table(const QConst& hq) {
    const int LW = int(hq.LW), L = int(hq.L), k = int(hq.k);
    const int NC = crt_tc_cols(LW);
    std::vector<uint8_t> b(crt_tc_table_bytes(LW), 0);
    for (int c = 0; c < NC; ++c)
        for (int i = 0; i < k; ++i)
            for (int a = 0; a < 8; ++a) {
                const int byte = c - a;
                if (byte < 0 || byte >= 4 * L) continue;
                const uint32_t word = hq.mq[size_t(i) * kMqStride + size_t(byte / 4)];
                const int K = 8 * i + a;
                b[size_t(c / 8) * 2048 + size_t(K / 16) * 128 + size_t(c % 8) * 16 + size_t(K % 16)] =
                    uint8_t(word >> (8 * (byte % 4)));
            }
    return b;
}

// The same table for the 30-bit engine: K byte 4 i + a (a < 4) of output column c holds byte
// c - a of (M/p_i) mod q.
std::vector<uint8_t> crt_tc32_table(const QConst32& hq) {
    const int LW = int(hq.LW), L = int(hq.L), k = int(hq.k);
    const int NC = crt_tc_cols(LW);
    std::vector<uint8_t> b(crt_tc_table_bytes(LW), 0);
    for (int c = 0; c < NC; ++c)
        for (int i = 0; i < k; ++i)
            for (int a = 0; a < 4; ++a) {
                const int byte = c - a;
                if (byte < 0 || byte >= 4 * L) continue;
                const uint32_t word = hq.mq[size_t(i) * kMqStride + size_t(byte / 4)];
                const int K = 4 * i + a;
                b[size_t(c / 8) * 2048 + size_t(K / 16) * 128 + size_t(c % 8) * 16 + size_t(K % 16)] =
                    uint8_t(word >> (8 * (byte % 4)));
            }
    return b;
}

bool word64_forced() {
    const char* word = std::getenv("NC_WORD_BITS");
    return word && std::atoi(word) == 64;
}

// Row configuration of the 30-bit engine before any tuning: blocks of 2^11 with radix-8 passes
// where N allows them, else the largest radix-16 block.
RowConfig default_row_config32(int logN) {
    RowConfig c{logN < 11 ? logN : 11, 3, 256};
    if (!row_config_valid(logN, c) || !row32_kernel(c)) c = RowConfig{logN < kRowLogMax ? logN : kRowLogMax, 4, 256};
    return c;
}

}  // namespace

static int copy_threads() {
    if (const char* s = std::getenv("NC_COPY_THREADS")) {
        const int v = std::atoi(s);
        if (v >= 1 && v <= 64) return v;
    }
    const int hc = int(std::thread::hardware_concurrency());
    return hc < 2 ? 1 : (hc < 8 ? hc : 8);
}

Plan* plan_create(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int factors) {
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
    p->factors = factors;
    const std::string err = build_qconst(q, int(L), logN, &p->hq, factors);
    if (!err.empty()) {
        delete p;
        throw Error(kEInval, err);
    }
    p->W = W ? int(W) : int(p->hq.qbits);
    if (W != 0 && (W < p->hq.qbits || (W + 31) / 32 != L)) {
        delete p;
        throw Error(kEInval, "W must be the bit width of q and L = (W + 31) / 32");
    }
    const std::string qerr = check_qconst(p->hq);
    if (!qerr.empty()) {
        delete p;
        throw Error(kESelfCheck, "init self-check of the plan's constants: " + qerr);
    }
    p->k = int(p->hq.k);
    if (!tuned_row_config(logN, int(L), &p->cfg)) p->cfg = default_row_config(logN);
    // the 30-bit engine: pairs whose bound fits its 64 primes
    bool w32_consts = false;
    if (factors == 2 && build_qconst32(q, int(L), logN, &p->hq32).empty()) {
        const std::string e32 = check_qconst32(p->hq32);
        if (!e32.empty()) {
            delete p;
            throw Error(kESelfCheck, "init self-check of the plan's 30-bit constants: " + e32);
        }
        w32_consts = true;
        p->k32 = int(p->hq32.k);
    }
    p->cfg32 = default_row_config32(logN);
    bool tuned_w32 = false;
    const bool tuned = tuned_engine(logN, int(L), &p->cfg32, &tuned_w32);
    try {
        p->device = current_device();
        p->tables = acquire_tables(p->device);
        if (!p->tables->tensor_cores) p->res_tc = p->crt_tc = false;  // integer-pipe engines only
        check(cudaMalloc(&p->d_qc, sizeof(QConst)), "plan constants");
        check(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "stream");
        // ordered on the plan's stream and complete before any other stream can use the plan
        check(cudaMemcpyAsync(p->d_qc, &p->hq, sizeof(QConst), cudaMemcpyHostToDevice, p->stream),
              "plan constants upload");
        std::vector<uint8_t> crt_b;
        if (p->k <= kCrtTcMaxPrimes) {
            crt_b = crt_tc_table(p->hq);
            check(cudaMalloc(&p->d_crt_b, crt_b.size()), "CRT table");
            check(cudaMemcpyAsync(p->d_crt_b, crt_b.data(), crt_b.size(), cudaMemcpyHostToDevice, p->stream),
                  "CRT table upload");
        }
        std::vector<uint8_t> crt_b32;
        if (w32_consts && p->tables->tensor_cores) {
            check(cudaMalloc(&p->d_qc32, sizeof(QConst32)), "30-bit plan constants");
            check(cudaMemcpyAsync(p->d_qc32, &p->hq32, sizeof(QConst32), cudaMemcpyHostToDevice, p->stream),
                  "30-bit plan constants upload");
            crt_b32 = crt_tc32_table(p->hq32);
            check(cudaMalloc(&p->d_crt_b32, crt_b32.size()), "30-bit CRT table");
            check(cudaMemcpyAsync(p->d_crt_b32, crt_b32.data(), crt_b32.size(), cudaMemcpyHostToDevice, p->stream),
                  "30-bit CRT table upload");
            p->w32_ok = true;
            // NC_WORD_BITS=64 keeps the 62-bit engine; otherwise the engine an autotune of this
            // (N, L) picked earlier in the process, else the 30-bit engine
            p->w32 = !word64_forced() && (tuned ? tuned_w32 : true);
        }
        check(cudaStreamSynchronize(p->stream), "plan constants upload");
        check(cudaEventCreate(&p->ev_start), "event");
        check(cudaEventCreate(&p->ev_stop), "event");
        if (const char* tr = std::getenv("NC_TRACE")) p->trace = tr[0] == '1';
        if (p->trace)
            for (auto& ev : p->ev_trace) check(cudaEventCreate(&ev), "event");
        for (auto& ev : p->ev_stage) check(cudaEventCreate(&ev), "event");
        device_self_test(p->device);
    } catch (...) {
        plan_destroy(p);
        throw;
    }
    return p;
}

namespace {
std::mutex g_selftest_mu;
std::map<int, int> g_selftest;  // device -> 1 while its self-test runs, 2 once it passed
}  // namespace

// Once per device, before the first plan there is handed out: an N = 8 product modulo
// q = 2^127 - 1 with 0, 1 and q - 1 among its coefficients, by the 30-bit engine and the 62-bit
// tensor-core stages (where the device has tensor cores) and by the 62-bit integer-pipe stages,
// compared with the host schoolbook. The plan it creates runs no self-test of its own.
void device_self_test(int device) {
    {
        std::lock_guard<std::mutex> lock(g_selftest_mu);
        int& st = g_selftest[device];
        if (st != 0) return;
        st = 1;
    }
    constexpr int N = 8, L = 4;
    const uint32_t q[L] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0x7fffffffu};
    std::vector<uint32_t> a(N * L), b(N * L), want(N * L), got(N * L);
    uint64_t x = 0x243f6a8885a308d3ull;
    for (int i = 0; i < N * L; ++i) {
        x = x * 6364136223846793005ull + 1442695040888963407ull;
        a[size_t(i)] = uint32_t(x >> 32);
        b[size_t(i)] = uint32_t(x >> 7);
    }
    for (int c = 0; c < N; ++c) {  // below q: top limbs under 2^31 - 1
        a[size_t(c) * L + 3] &= 0x7ffffffeu;
        b[size_t(c) * L + 3] &= 0x7ffffffeu;
    }
    for (int l = 0; l < L; ++l) {
        a[size_t(1) * L + l] = q[l] - (l == 0 ? 1u : 0u);  // q - 1
        b[size_t(2) * L + l] = q[l] - (l == 0 ? 1u : 0u);
        a[size_t(3) * L + l] = 0;
        b[size_t(5) * L + l] = l == 0 ? 1u : 0u;
    }
    schoolbook_negacyclic(N, L, q, a.data(), b.data(), want.data());
    Plan* p = nullptr;
    uint32_t* d = nullptr;
    std::string err;
    try {
        p = plan_create(N, 0, L, q);
        check(cudaMalloc(&d, size_t(3) * N * L * 4), "self-test buffers");
        check(cudaMemcpy(d, a.data(), size_t(N) * L * 4, cudaMemcpyHostToDevice), "self-test upload");
        check(cudaMemcpy(d + N * L, b.data(), size_t(N) * L * 4, cudaMemcpyHostToDevice), "self-test upload");
        // engines: the 30-bit one (where the device has it), the 62-bit tensor-core stages, the
        // 62-bit integer-pipe stages
        const char* names[3] = {"30-bit", "default 62-bit", "integer-pipe 62-bit"};
        for (int engines = p->w32_ok ? 0 : 1; engines < 3 && err.empty(); ++engines) {
            p->w32 = engines == 0;
            if (engines == 2) p->res_tc = p->crt_tc = false;
            check(cudaMemsetAsync(d + 2 * N * L, 0xff, size_t(N) * L * 4, p->stream), "self-test output");
            plan_multiply_device(p, d, d + N * L, d + 2 * N * L, p->stream);
            check(cudaStreamSynchronize(p->stream), "self-test product");
            check(cudaMemcpy(got.data(), d + 2 * N * L, size_t(N) * L * 4, cudaMemcpyDeviceToHost), "self-test download");
            if (got != want) err = std::string("the ") + names[engines] + " stages' N = 8 product differs from the schoolbook";
        }
    } catch (...) {
        cudaFree(d);
        plan_destroy(p);
        std::lock_guard<std::mutex> lock(g_selftest_mu);
        g_selftest[device] = 0;
        throw;
    }
    cudaFree(d);
    plan_destroy(p);
    std::lock_guard<std::mutex> lock(g_selftest_mu);
    g_selftest[device] = err.empty() ? 2 : 0;
    if (!err.empty()) throw Error(kESelfCheck, "device self-test: " + err);
}

// The plain path's residue scratch (k N u64 or k32 N u32 per operand, whichever is larger),
// allocated on its first use: plans used only inside batches or through the allocation-free
// entry point never hold it.
void ensure_scratch(Plan* p) {
    if (p->d_ra) return;
    const size_t res = p->residue_bytes();
    uint64_t* bufs[kMaxFactors] = {};
    for (int f = 0; f < p->factors; ++f) {
        const cudaError_t e = cudaMalloc(&bufs[f], res);
        if (e != cudaSuccess) {
            for (int g = 0; g < f; ++g) cudaFree(bufs[g]);
            check(e, "residue scratch");
        }
    }
    p->d_rb = bufs[1];
    for (int f = 2; f < p->factors; ++f) p->d_rx[f - 2] = bufs[f];
    p->d_ra = bufs[0];
}

// Staging for host operands (device copies, pinned buffers, copy threads), on first use.
void ensure_host_path(Plan* p) {
    ensure_scratch(p);
    if (p->pool) return;
    const size_t limbs = p->limbs() * sizeof(uint32_t);
    check(cudaMalloc(&p->d_a, limbs), "input a");
    check(cudaMalloc(&p->d_b, limbs), "input b");
    check(cudaMalloc(&p->d_c, limbs), "output c");
    check(cudaMallocHost(&p->h_a, limbs), "pinned a");
    check(cudaMallocHost(&p->h_b, limbs), "pinned b");
    check(cudaMallocHost(&p->h_c, limbs), "pinned c");
    check(cudaMalloc(&p->d_hat, p->residue_bytes()), "operand a in the NTT domain");
    for (int f = 2; f < p->factors; ++f) {
        check(cudaMalloc(&p->d_x[f - 2], limbs), "input operand");
        check(cudaMallocHost(&p->h_x[f - 2], limbs), "pinned operand");
    }
    // one set of copy threads per process, shared by every plan (jobs run one at a time)
    static HostPool* shared = new HostPool(copy_threads());
    p->ev_out.assign(size_t(kMaxOutChunks), nullptr);
    for (auto& ev : p->ev_out) check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
    p->ev_grp.assign(4, nullptr);
    for (auto& ev : p->ev_grp) check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
    check(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking), "copy stream");
    check(cudaEventCreateWithFlags(&p->ev_a, cudaEventDisableTiming), "event");
    check(cudaEventCreateWithFlags(&p->ev_b, cudaEventDisableTiming), "event");
    p->pool = shared;
}

void plan_destroy(Plan* p) {
    if (!p) return;
    if (p->copy_stream) cudaStreamSynchronize(p->copy_stream);
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    if (p->ev_a) cudaEventDestroy(p->ev_a);
    if (p->ev_b) cudaEventDestroy(p->ev_b);
    cudaFree(p->d_qc);
    cudaFree(p->d_crt_b);
    cudaFree(p->d_qc32);
    cudaFree(p->d_crt_b32);
    cudaFree(p->d_ra);
    cudaFree(p->d_rb);
    cudaFree(p->d_hat);
    for (int f = 0; f < kMaxFactors - 2; ++f) {
        cudaFree(p->d_rx[f]);
        cudaFree(p->d_x[f]);
        cudaFreeHost(p->h_x[f]);
    }
    cudaFree(p->d_a);
    cudaFree(p->d_b);
    cudaFree(p->d_c);
    cudaFreeHost(p->h_a);
    cudaFreeHost(p->h_b);
    cudaFreeHost(p->h_c);
    if (p->ev_start) cudaEventDestroy(p->ev_start);
    if (p->ev_stop) cudaEventDestroy(p->ev_stop);
    for (auto ev : p->ev_trace)
        if (ev) cudaEventDestroy(ev);
    for (auto ev : p->ev_stage)
        if (ev) cudaEventDestroy(ev);
    if (p->stream) cudaStreamDestroy(p->stream);
    for (auto ev : p->ev_out)
        if (ev) cudaEventDestroy(ev);
    for (auto ev : p->ev_grp)
        if (ev) cudaEventDestroy(ev);
    release_tables(p->tables);
    delete p;
}

void plan_multiply_device(Plan* p, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t stream) {
    if (!p) throw Error(kEInval, "null plan");
    if (!d_a || !d_b || !d_c) throw Error(kEInval, "null device buffer");
    if (((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_b) | reinterpret_cast<uintptr_t>(d_c)) &
         15) != 0)
        throw Error(kEInval, "device buffers must be 16-byte aligned");
    ensure_scratch(p);
    const ProductDesc d = p->desc_plain(d_a, d_b, d_c);
    check(launch_product(d, p->tables->view(), p->plain_cfg(), stream, p->timing ? p->ev_stage : nullptr),
          "kernel launch");
}

namespace {

// [lo, hi) of part `part` out of `parts` for `bytes`, in 4 KiB granules.
void slice(size_t bytes, int part, int parts, size_t* lo, size_t* hi) {
    const size_t granules = (bytes + 4095) / 4096;
    const size_t per = (granules + size_t(parts) - 1) / size_t(parts);
    *lo = std::min(bytes, per * size_t(part) * 4096);
    *hi = std::min(bytes, per * size_t(part + 1) * 4096);
}

// Host-to-device copies of a few MB each: on PCIe 5 hosts, copies of a few hundred KB reach well
// under half the link rate (per-copy overhead), and multi-MB copies reach most of it. The first
// operand's chunks grow from 512 KB (512 KB, 1, 2, 4, 4 ... MB): the link idles only while the
// first, small chunk is staged (staging runs at about 1.8 times the link rate, so each chunk is
// staged while the one before it transfers), where one 4 MB first chunk left it idle ~40 us.
constexpr size_t kDmaChunk = size_t(4) << 20;
constexpr size_t kFirstChunk = size_t(512) << 10;

std::vector<std::pair<size_t, size_t>> upload_chunks(size_t bytes, bool ramp) {
    std::vector<std::pair<size_t, size_t>> out;
    size_t want = ramp ? kFirstChunk : kDmaChunk;
    for (size_t off = 0; off < bytes;) {
        size_t len = std::min(want, bytes - off);
        if (bytes - off - len < want / 2) len = bytes - off;  // no small last chunk
        out.emplace_back(off, len);
        off += len;
        want = std::min(kDmaChunk, 2 * want);
    }
    return out;
}

// The product comes back in device-to-host copies that shrink towards the end (the rest, then
// 2.5 MB pieces, 1 MB, 384 KB; one event each): every chunk's copy-out into the caller's buffer
// overlaps the next chunk's transfer, so what follows the last transfer is the copy-out of a
// 384 KB chunk (three equal 2.5 MB chunks left ~40 us of copy-out after the last one landed;
// chunks of 1 MB and less transfer at only 30-40 GB/s, so the others stay large).
std::vector<std::pair<size_t, size_t>> download_chunks(size_t bytes) {
    std::vector<size_t> lens;  // from the last chunk backwards
    const size_t tail[] = {size_t(384) << 10, size_t(1) << 20};
    size_t left = bytes;
    for (size_t t : tail) {
        if (left <= t + (t >> 1)) break;
        lens.push_back(t);
        left -= t;
    }
    const size_t piece = size_t(5) << 19;
    while (left > piece + (piece >> 1) && int(lens.size()) < kMaxOutChunks - 1) {
        lens.push_back(piece);
        left -= piece;
    }
    if (left) lens.push_back(left);
    std::vector<std::pair<size_t, size_t>> out;
    size_t off = 0;
    for (auto it = lens.rbegin(); it != lens.rend(); ++it) {
        out.emplace_back(off, *it);
        off += *it;
    }
    return out;
}

// Operand b of a pair goes up in this many column groups, each a strided copy of its columns of
// every row segment, and each group's residue tiles start as soon as it has landed: the residue
// stage of b then ends about one group's tiles after the last byte, not a whole stage after.
int upload_groups(const Plan* p, const ProductDesc& d) {
    constexpr int kGroups = 4;
    if (p->N < (1 << 13)) return 1;
    return residue_tiles(d, p->plain_cfg()) % kGroups == 0 ? kGroups : 1;
}

}  // namespace

namespace {

// Host operands x[0..n) of the plan's product (n = 2, or the plan's factors for a chain).
void submit_host_operands(Plan* p, const uint32_t* const* x, int n) {
    if (!p) throw Error(kEInval, "null plan");
    for (int f = 0; f < n; ++f)
        if (!x[f]) throw Error(kEInval, "null host buffer");
    ensure_host_path(p);
    const size_t bytes = p->limbs() * sizeof(uint32_t);
    // Each operand goes in chunks: every copy thread stages its part of a chunk into pinned memory,
    // then the chunk's DMA is enqueued and runs while the next chunk is staged. Operand a goes on
    // the plan's stream; operand b on the copy stream, after a's upload (so a arrives first at full
    // link rate), and a's stages run while b uploads.
    const char* srcs[kMaxFactors];
    char* pins[kMaxFactors];
    char* devs[kMaxFactors];
    uint32_t* dev_ops[kMaxFactors];
    for (int f = 0; f < n; ++f) {
        srcs[f] = reinterpret_cast<const char*>(x[f]);
        uint32_t* pin = f == 0 ? p->h_a : f == 1 ? p->h_b : p->h_x[f - 2];
        dev_ops[f] = f == 0 ? p->d_a : f == 1 ? p->d_b : p->d_x[f - 2];
        pins[f] = reinterpret_cast<char*>(pin);
        devs[f] = reinterpret_cast<char*>(dev_ops[f]);
    }
    ProductDesc d = n == 2 ? p->desc_plain(p->d_a, p->d_b, p->d_c) : p->desc_chain(dev_ops, p->d_c);
    int groups = 1;  // column groups of b's upload (pairs only)
    const bool trace = p->trace && n == 2;
    auto since = [p] {
        return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - p->trace_t0).count();
    };
    if (trace) {
        p->trace_t0 = std::chrono::steady_clock::now();
        check(cudaEventRecord(p->ev_trace[0], p->stream), "event");
    }
    for (int op = 0; op < n; ++op) {
        cudaStream_t stream = op == 0 ? p->stream : p->copy_stream;
        if (op == 1) {
            // b's buffers may still be read by the plan's stream (a previous product): order the
            // copy stream after everything enqueued there so far, including a's upload
            check(cudaEventRecord(p->ev_a, p->stream), "event");
            // a's stages go on the plan's stream now, before any copy of the other operands is
            // queued: work queued on that stream behind a's upload after those copies were queued
            // waited for them (measured: the kernel started only once b had landed). For a pair,
            // that is a's residues and forward transforms (the GPU is otherwise idle while b
            // uploads), and the product then takes a in the NTT domain; for a chain, a's residues.
            check(cudaEventRecord(p->ev_start, p->stream), "event");
            if (p->timing) check(cudaEventRecord(p->ev_stage[0], p->stream), "event");
            if (n == 2) {
                ProductDesc fa = d;
                fa.mode = kModeForward;
                fa.b = nullptr;
                fa.c = nullptr;
                fa.hat_out = p->d_hat;
                if (trace) {
                    p->trace_host[0] = since();
                    check(cudaEventRecord(p->ev_trace[1], p->stream), "event");
                }
                check(launch_product(fa, p->tables->view(), p->plain_cfg(), p->stream), "kernel launch");
                if (trace) check(cudaEventRecord(p->ev_trace[2], p->stream), "event");
                d.mode = kModeCachedA;
                d.a = nullptr;
                d.a_hat = p->d_hat;
                groups = upload_groups(p, d);
            } else {
                check(launch_residues(d, p->tables->view(), p->plain_cfg(), p->stream, 0, 1), "kernel launch");
            }
            check(cudaStreamWaitEvent(p->copy_stream, p->ev_a, 0), "stream wait");
        }
        if (op == 1 && groups > 1) {
            // group g is columns [g N2 / G, (g + 1) N2 / G) of every row segment: the copy threads
            // stage its N1 pieces, then one strided copy takes it up and its residue tiles follow on
            // the plan's stream, so on a host whose staging is slower than the link b's transfer
            // starts after a quarter of b is staged, not all of it
            const int N1 = 1 << (p->logN - p->plain_cfg().logN2);
            const size_t N2 = size_t(1) << p->plain_cfg().logN2, row = N2 * size_t(p->L) * 4;
            const size_t width = row / size_t(groups);
            for (int g = 0; g < groups; ++g) {
                const size_t col = size_t(g) * width;
                p->pool->run([&](int part, int parts) {
                    for (int u = part; u < N1; u += parts)
                        stage_copy(pins[op] + size_t(u) * row + col, srcs[op] + size_t(u) * row + col, width);
                });
                check(cudaMemcpy2DAsync(devs[op] + col, row, pins[op] + col, row, width, size_t(N1),
                                        cudaMemcpyHostToDevice, stream),
                      "operand copy");
                check(cudaEventRecord(p->ev_grp[size_t(g)], stream), "event");
            }
            continue;
        }
        for (const auto& ch : upload_chunks(bytes, op == 0)) {
            const size_t off = ch.first, len = ch.second;
            p->pool->run([&](int part, int parts) {
                size_t lo, hi;
                slice(len, part, parts, &lo, &hi);
                if (hi > lo) stage_copy(pins[op] + off + lo, srcs[op] + off + lo, hi - lo);
            });
            check(cudaMemcpyAsync(devs[op] + off, pins[op] + off, len, cudaMemcpyHostToDevice, stream),
                  "operand copy");
        }
    }
    check(cudaEventRecord(p->ev_b, p->copy_stream), "event");
    if (trace) {
        p->trace_host[1] = since();
        check(cudaEventRecord(p->ev_trace[3], p->copy_stream), "event");
    }
    if (groups > 1) {
        if (p->timing) check(cudaEventRecord(p->ev_stage[0], p->stream), "event");
        for (int g = 0; g < groups; ++g) {
            check(cudaStreamWaitEvent(p->stream, p->ev_grp[size_t(g)], 0), "stream wait");
            check(launch_residues(d, p->tables->view(), p->plain_cfg(), p->stream, 1, 1, g, groups), "kernel launch");
        }
        cudaEvent_t* ev = p->timing ? p->ev_stage : nullptr;
        check(launch_product(d, p->tables->view(), p->plain_cfg(), p->stream, ev, nullptr, true), "kernel launch");
    } else {
        check(launch_product(d, p->tables->view(), p->plain_cfg(), p->stream, p->timing ? p->ev_stage : nullptr, p->ev_b),
              "kernel launch");
    }
    check(cudaEventRecord(p->ev_stop, p->stream), "event");
    if (trace) check(cudaEventRecord(p->ev_trace[4], p->stream), "event");
    const auto out = download_chunks(bytes);
    for (size_t j = 0; j < out.size(); ++j) {
        check(cudaMemcpyAsync(reinterpret_cast<char*>(p->h_c) + out[j].first,
                              reinterpret_cast<char*>(p->d_c) + out[j].first, out[j].second, cudaMemcpyDeviceToHost,
                              p->stream),
              "product copy");
        check(cudaEventRecord(p->ev_out[j], p->stream), "event");
    }
    if (trace) {
        check(cudaEventRecord(p->ev_trace[5], p->stream), "event");
        p->trace_host[2] = since();
    }
}

}  // namespace

void plan_submit_host(Plan* p, const uint32_t* a, const uint32_t* b) {
    const uint32_t* x[2] = {a, b};
    submit_host_operands(p, x, 2);
}

void plan_collect_host(Plan* p, uint32_t* c) {
    if (!p) throw Error(kEInval, "null plan");
    if (!c) throw Error(kEInval, "null host buffer");
    if (!p->pool) throw Error(kEInval, "collect without a submitted product");
    const size_t bytes = p->limbs() * sizeof(uint32_t);
    const auto out = download_chunks(bytes);
    const int nd = int(out.size());
    std::atomic<int> err{int(cudaSuccess)};
    // Every copy thread takes its share of each chunk as soon as that chunk has landed, so the
    // copy-out after the last transfer is one chunk split over all threads. Only the calling
    // thread asks the driver (polling the chunk's event) and publishes the count of landed chunks;
    // the others spin on that count: eight threads waiting on one event in the driver saw each
    // chunk 20-30 us late and apart.
    std::atomic<int> landed{0};
    p->pool->run([&](int part, int parts) {
        for (int j = 0; j < nd; ++j) {
            if (part == 0) {
                cudaError_t e;
                while ((e = cudaEventQuery(p->ev_out[size_t(j)])) == cudaErrorNotReady) {
                }
                if (e != cudaSuccess) {
                    err.store(int(e));
                    landed.store(nd + 1, std::memory_order_release);  // releases the other threads
                    return;
                }
                landed.store(j + 1, std::memory_order_release);
            } else {
                int seen;
                while ((seen = landed.load(std::memory_order_acquire)) <= j) {
                }
                if (seen > nd) return;
            }
            const size_t base = out[size_t(j)].first, n = out[size_t(j)].second;
            size_t lo, hi;
            slice(n, part, parts, &lo, &hi);
            if (hi > lo)
                stage_copy(reinterpret_cast<char*>(c) + base + lo, reinterpret_cast<const char*>(p->h_c) + base + lo,
                           hi - lo);
        }
    });
    check(cudaError_t(err.load()), "product");
    // the last output chunk's event is the last work of the product on the plan's stream
    cudaEventElapsedTime(&p->last_kernel_ms, p->ev_start, p->ev_stop);
    if (p->trace) {
        // one line per call: device-clock phase ends (from the call's start event) and host times
        p->trace_host[3] = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - p->trace_t0).count();
        float g[5] = {0, 0, 0, 0, 0};
        for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&g[i], p->ev_trace[0], p->ev_trace[i + 1]);
        std::fprintf(stderr,
                     "nc_trace a_uploaded=%.1f a_forward=%.1f b_uploaded=%.1f product=%.1f downloaded=%.1f "
                     "a_staged=%.1f b_staged=%.1f enqueued=%.1f collected=%.1f\n",
                     1e3 * g[0], 1e3 * g[1], 1e3 * g[2], 1e3 * g[3], 1e3 * g[4], p->trace_host[0], p->trace_host[1],
                     p->trace_host[2], p->trace_host[3]);
    }
}

void plan_multiply_host(Plan* p, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    plan_submit_host(p, a, b);
    plan_collect_host(p, c);
}

void plan_multiply_chain_host(Plan* p, const uint32_t* const* x, uint32_t* c) {
    if (!p) throw Error(kEInval, "null plan");
    if (!x) throw Error(kEInval, "null operand list");
    submit_host_operands(p, x, p->factors);
    plan_collect_host(p, c);
}

void plan_multiply_chain_device(Plan* p, const uint32_t* const* d_x, uint32_t* d_c, cudaStream_t stream) {
    if (!p) throw Error(kEInval, "null plan");
    if (!d_x || !d_c) throw Error(kEInval, "null device buffer");
    uintptr_t align = reinterpret_cast<uintptr_t>(d_c);
    for (int f = 0; f < p->factors; ++f) {
        if (!d_x[f]) throw Error(kEInval, "null device buffer");
        align |= reinterpret_cast<uintptr_t>(d_x[f]);
    }
    if (align & 15) throw Error(kEInval, "device buffers must be 16-byte aligned");
    ensure_scratch(p);
    check(launch_product(p->desc_chain(d_x, d_c), p->tables->view(), p->cfg, stream,
                         p->timing ? p->ev_stage : nullptr),
          "kernel launch");
}

// ------------------------------------------------------------------------------ row configuration

namespace {
std::mutex g_tune_mu;
std::map<std::pair<int, int>, RowConfig> g_tuned;  // the 62-bit engine's row configuration
struct Tuned32 {
    RowConfig cfg;  // the 30-bit engine's row configuration
    bool use;       // it was the faster engine
};
std::map<std::pair<int, int>, Tuned32> g_tuned32;
}  // namespace

bool tuned_row_config(int logN, int L, RowConfig* out) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find({logN, L});
    if (it == g_tuned.end()) return false;
    *out = it->second;
    return true;
}

bool tuned_engine(int logN, int L, RowConfig* cfg32, bool* use_w32) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned32.find({logN, L});
    if (it == g_tuned32.end()) return false;
    *cfg32 = it->second.cfg;
    *use_w32 = it->second.use;
    return true;
}

void plan_set_row_config(Plan* p, const RowConfig& c) {
    if (!p) throw Error(kEInval, "null plan");
    if (p->use_w32()) {
        if (!row_config_valid(p->logN, c) || !row32_kernel(c))
            throw Error(kEInval, "no compiled 30-bit row kernel for this configuration and N");
        p->cfg32 = c;
        return;
    }
    if (!row_config_valid(p->logN, c) || !row_variant_exists(c))
        throw Error(kEInval, "no compiled row kernel for this configuration and N");
    p->cfg = c;
}

void plan_set_word_bits(Plan* p, int bits) {
    if (!p) throw Error(kEInval, "null plan");
    if (bits == 64) {
        p->w32 = false;
        return;
    }
    if (bits != 32) throw Error(kEInval, "word bits must be 32 or 64");
    if (!p->w32_ok)
        throw Error(kEInval,
                    "the 30-bit engine needs tensor cores, a product of two operands and a bound within 64 primes "
                    "below 2^30");
    p->w32 = true;
}

float plan_autotune(Plan* p, int reps) {
    if (!p) throw Error(kEInval, "null plan");
    if (reps < 1) reps = 1;
    ensure_host_path(p);
    // Operands: the plan's own staging buffers with reduced random limbs (values need not be < q
    // for timing; every limb pattern runs the same instructions).
    const size_t words = p->limbs();
    std::vector<uint32_t> host(words);
    uint64_t s = 0x9E3779B97F4A7C15ull;
    for (size_t w = 0; w < words; ++w) {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        host[w] = uint32_t(s);
    }
    for (size_t n = 0; n < size_t(p->N); ++n) host[n * p->L + p->L - 1] &= p->hq.q[p->L - 1] >> 1;
    check(cudaMemcpyAsync(p->d_a, host.data(), words * 4, cudaMemcpyHostToDevice, p->stream), "tune upload");
    check(cudaMemcpyAsync(p->d_b, host.data(), words * 4, cudaMemcpyHostToDevice, p->stream), "tune upload");
    check(cudaStreamSynchronize(p->stream), "tune upload");
    auto time_product = [&](const RowConfig& c) {
        const ProductDesc d = p->desc_plain(p->d_a, p->d_b, p->d_c);
        check(launch_product(d, p->tables->view(), c, p->stream), "tune launch");  // warm-up
        check(cudaEventRecord(p->ev_start, p->stream), "event");
        for (int r = 0; r < reps; ++r) check(launch_product(d, p->tables->view(), c, p->stream), "tune launch");
        check(cudaEventRecord(p->ev_stop, p->stream), "event");
        check(cudaEventSynchronize(p->ev_stop), "tune");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, p->ev_start, p->ev_stop), "event");
        return ms / float(reps);
    };
    // the 62-bit engine's row configurations
    const bool was_w32 = p->w32;
    p->w32 = false;
    RowConfig best = p->cfg;
    float best_ms = 1e30f;
    for (const RowConfig& c : row_variants(p->logN)) {
        p->cfg = c;
        const float ms = time_product(c);
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    p->cfg = best;
    // the 30-bit engine's, where it can run; the faster engine is kept
    const bool try32 = p->w32_ok && p->res_tc && p->crt_tc && !word64_forced();
    RowConfig best32 = p->cfg32;
    float best32_ms = 1e30f;
    if (try32) {
        p->w32 = true;
        for (const RowConfig& c : all_row32_variants()) {
            if (!row_config_valid(p->logN, c)) continue;
            p->cfg32 = c;
            const float ms = time_product(c);
            if (ms < best32_ms) {
                best32_ms = ms;
                best32 = c;
            }
        }
        p->cfg32 = best32;
        p->w32 = best32_ms < best_ms;
    } else {
        p->w32 = was_w32;
    }
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[{p->logN, p->L}] = best;
    if (try32) g_tuned32[{p->logN, p->L}] = Tuned32{best32, p->w32};
    return try32 && best32_ms < best_ms ? best32_ms : best_ms;
}

}  // namespace nc
