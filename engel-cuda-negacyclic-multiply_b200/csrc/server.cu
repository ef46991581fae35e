// Serving loop (see server.h).
#include "server.h"

#include "hostcopy.h"

#include <algorithm>
#include <chrono>
#include <cstring>

namespace nc {

namespace {

constexpr size_t kGranule = 256;

size_t granules(size_t bytes) { return (bytes + kGranule - 1) / kGranule * kGranule; }

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// ------------------------------------------------------------------ arena

void Arena::reset(char* base, size_t bytes) {
    base_ = base;
    bytes_ = bytes / kGranule * kGranule;
    in_use_ = 0;
    free_.clear();
    used_.clear();
    if (bytes_) free_[0] = bytes_;
}

char* Arena::alloc(size_t bytes) {
    const size_t need = granules(bytes ? bytes : 1);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < need) continue;
        const size_t off = it->first, size = it->second;
        free_.erase(it);
        if (size > need) free_[off + need] = size - need;
        used_[off] = need;
        in_use_ += need;
        return base_ + off;
    }
    return nullptr;
}

void Arena::free(char* p) {
    if (!p) return;
    const size_t off = size_t(p - base_);
    auto u = used_.find(off);
    if (u == used_.end()) return;
    size_t start = off, size = u->second;
    in_use_ -= size;
    used_.erase(u);
    auto next = free_.lower_bound(start);
    if (next != free_.end() && next->first == start + size) {
        size += next->second;
        free_.erase(next);
    }
    auto prev = free_.lower_bound(start);
    if (prev != free_.begin()) {
        --prev;
        if (prev->first + prev->second == start) {
            start = prev->first;
            size += prev->second;
            free_.erase(prev);
        }
    }
    free_[start] = size;
}

// ------------------------------------------------------------------ server

Server::Server(int device, size_t hbm_budget, size_t staging_bytes, int max_batch, int streams)
    : device_(device), max_batch_(std::max(1, max_batch)) {
    if (hbm_budget < (size_t(1) << 20) || staging_bytes < (size_t(1) << 20))
        throw Error(kEInval, "budgets must be at least 1 MiB");
    if (streams < 1 || streams > 16) throw Error(kEInval, "streams must be 1..16");
    try {
        check(cudaMalloc(&dev_base_, hbm_budget), "server HBM budget");
        check(cudaMallocHost(&host_base_, staging_bytes), "server pinned staging");
        dev_arena_.reset(dev_base_, hbm_budget);
        host_arena_.reset(host_base_, staging_bytes);
        for (int s = 0; s < streams; ++s) {
            cudaStream_t st = nullptr;
            check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "server stream");
            streams_.push_back(st);
            batches_.emplace_back(new Batch(device));
            stream_busy_.push_back(false);
        }
        check(cudaEventCreate(&origin_), "event");
        check(cudaEventRecord(origin_, streams_[0]), "event");
    } catch (...) {
        if (origin_) cudaEventDestroy(origin_);
        for (auto s : streams_) cudaStreamDestroy(s);
        batches_.clear();
        cudaFree(dev_base_);
        cudaFreeHost(host_base_);
        throw;
    }
    thread_ = std::thread([this] { loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    if (thread_.joinable()) thread_.join();
    for (auto s : streams_) cudaStreamSynchronize(s);
    for (auto& f : flights_) {
        cudaEventDestroy(f.begin);
        cudaEventDestroy(f.done);
    }
    if (origin_) cudaEventDestroy(origin_);
    batches_.clear();
    for (auto s : streams_) cudaStreamDestroy(s);
    cudaFree(dev_base_);
    cudaFreeHost(host_base_);
}

int Server::register_operand(Plan* plan, const uint32_t* a) {
    if (!plan || !a) throw Error(kEInval, "null plan or operand");
    if (plan->device != device_ || current_device() != device_)
        throw Error(kEInval, "the plan and the calling thread must be on the server's device");
    const size_t limb = granules(plan->limbs() * 4);
    const size_t hat = granules(plan->residue_bytes());  // either engine's NTT-domain form
    const size_t scratch = 2 * hat;
    char *dev_hat, *tmp;
    {
        std::lock_guard<std::mutex> lock(mu_);
        dev_hat = dev_arena_.alloc(hat);
        tmp = dev_hat ? dev_arena_.alloc(limb + scratch) : nullptr;
        if (!tmp) {
            dev_arena_.free(dev_hat);
            throw Error(kENoMem, "the HBM budget cannot hold this operand");
        }
    }
    cudaStream_t s = nullptr;
    try {
        check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        {
            // the batch synchronises its last stream when destroyed, so it must go before s
            Batch fwd(device_);
            check(cudaMemcpyAsync(tmp, a, plan->limbs() * 4, cudaMemcpyHostToDevice, s), "operand copy");
            fwd.add(plan, kModeForward, reinterpret_cast<uint32_t*>(tmp), nullptr, nullptr, nullptr,
                    reinterpret_cast<uint64_t*>(dev_hat), reinterpret_cast<uint64_t*>(tmp + limb));
            fwd.run(s, false);
            fwd.synchronize();
        }
        cudaStreamDestroy(s);
    } catch (...) {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        std::lock_guard<std::mutex> lock(mu_);
        dev_arena_.free(tmp);
        dev_arena_.free(dev_hat);
        throw;
    }
    std::lock_guard<std::mutex> lock(mu_);
    dev_arena_.free(tmp);
    const int id = next_operand_++;
    operands_[id] = Operand{plan, dev_hat, hat};
    return id;
}

void Server::release_operand(int id) {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = operands_.find(id);
    if (it == operands_.end()) throw Error(kEInval, "unknown operand");
    if (it->second.pins > 0) throw Error(kEBusy, "the operand is used by a request being submitted");
    for (auto& kv : requests_)
        if (kv.second->operand == id && kv.second->status < 2 && kv.second->status >= 0)
            throw Error(kEBusy, "the operand is used by a pending request");
    dev_arena_.free(it->second.dev);
    operands_.erase(it);
}

uint64_t Server::submit(Plan* plan, const uint32_t* a, int operand, const uint32_t* b) {
    if (!plan || !b) throw Error(kEInval, "null plan or operand");
    if (plan->device != device_) throw Error(kEInval, "the plan lives on another device");
    auto r = std::make_unique<Request>();
    r->plan = plan;
    r->operand = operand;
    r->limb_bytes = granules(plan->limbs() * 4);
    r->dev_bytes = 3 * r->limb_bytes + 2 * granules(plan->residue_bytes());
    auto check_operand = [&]() -> std::map<int, Operand>::iterator {
        auto it = operands_.find(operand);
        if (it == operands_.end()) throw Error(kEInval, "unknown operand");
        if (it->second.plan->N != plan->N || it->second.plan->k != plan->k ||
            it->second.plan->use_w32() != plan->use_w32() ||
            std::memcmp(it->second.plan->hq.q, plan->hq.q, sizeof(plan->hq.q)) != 0)
            throw Error(kEInval, "the operand was registered for another N or q");
        return it;
    };
    {
        std::unique_lock<std::mutex> lock(mu_);
        if (!fault_.empty()) throw Error(kECuda, "server stopped after a device error: " + fault_);
        if (operand >= 0)
            check_operand();
        else if (!a)
            throw Error(kEInval, "null operand a");
        if (3 * r->limb_bytes > host_arena_.capacity() || r->dev_bytes > dev_arena_.capacity())
            throw Error(kENoMem, "the request is larger than the server's budgets");
        space_cv_.wait(lock, [&] { return (r->host = host_arena_.alloc(3 * r->limb_bytes)) != nullptr || stop_; });
        if (stop_) throw Error(kEBusy, "server is stopping");
        if (operand >= 0) {
            // the lock is dropped for the staging copies below: pin the operand so that
            // release_operand cannot free it before the request is queued (the wait above may
            // also have let a release through, so the operand is looked up again here)
            auto it = operands_.find(operand);
            if (it == operands_.end()) {
                host_arena_.free(r->host);
                space_cv_.notify_all();
                throw Error(kEInval, "unknown operand");
            }
            ++it->second.pins;
        }
        r->id = next_id_++;
    }
    const size_t bytes = plan->limbs() * 4;
    if (operand < 0) stage_copy(r->host, reinterpret_cast<const char*>(a), bytes);
    stage_copy(r->host + r->limb_bytes, reinterpret_cast<const char*>(b), bytes);
    std::lock_guard<std::mutex> lock(mu_);
    if (operand >= 0) --operands_.at(operand).pins;  // from here the queued request keeps it
    r->t_submit = now_ms();
    if (t_first_ < 0) t_first_ = r->t_submit;
    const uint64_t id = r->id;
    queue_.push_back(r.get());
    requests_[id] = std::move(r);
    cv_.notify_all();
    return id;
}

bool Server::done(uint64_t id) {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end()) throw Error(kEInval, "unknown request");
    return it->second->status == 2 || it->second->status < 0;
}

double Server::wait(uint64_t id, uint32_t* c) {
    std::unique_lock<std::mutex> lock(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end()) throw Error(kEInval, "unknown request");
    Request* r = it->second.get();
    done_cv_.wait(lock, [&] { return r->status == 2 || r->status < 0; });
    if (r->status < 0) {
        const int r_status = r->status;
        const bool memory = r_status == -3;
        host_arena_.free(r->host);
        requests_.erase(it);
        space_cv_.notify_all();
        if (memory) throw Error(kENoMem, "the HBM budget cannot hold this request beside the registered operands");
        if (r_status == -4) throw Error(kETimeout, "the request's batch failed: " + last_timeout_);
        throw Error(kECuda, "request failed: " + fault_);
    }
    const double latency = r->t_done - r->t_submit;
    char* src = r->host + 2 * r->limb_bytes;
    const size_t bytes = r->plan->limbs() * 4;
    lock.unlock();
    if (c) std::memcpy(c, src, bytes);
    lock.lock();
    host_arena_.free(r->host);
    requests_.erase(it);
    space_cv_.notify_all();
    return latency;
}

void Server::stats(double* p50_ms, double* p99_ms, uint64_t* completed, double* products_per_s, size_t* hbm_in_use,
                   uint64_t* batches, uint64_t* timeouts) {
    std::lock_guard<std::mutex> lock(mu_);
    std::vector<double> v = latencies_;
    auto pct = [&](double f) {
        if (v.empty()) return 0.0;
        const size_t k = std::min(v.size() - 1, size_t(f * double(v.size() - 1) + 0.5));
        std::nth_element(v.begin(), v.begin() + long(k), v.end());
        return v[k];
    };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (completed) *completed = latencies_.size();
    if (products_per_s)
        *products_per_s = (latencies_.empty() || t_last_ <= t_first_) ? 0.0
                                                                        : 1e3 * double(latencies_.size()) / (t_last_ - t_first_);
    if (hbm_in_use) *hbm_in_use = dev_arena_.in_use();
    if (batches) *batches = batches_run_;
    if (timeouts) *timeouts = timeouts_;
}

void Server::io_stats(uint64_t* h2d_bytes, uint64_t* d2h_bytes, double* busy_ms, double* window_ms,
                      double* scheduler_ms) {
    std::lock_guard<std::mutex> lock(mu_);
    std::vector<std::pair<double, double>> v = busy_;
    std::sort(v.begin(), v.end());
    double busy = 0, lo = 0, hi = 0, first = 0, last = 0;
    bool open = false;
    for (const auto& iv : v) {
        if (!open) {
            lo = iv.first;
            hi = iv.second;
            first = iv.first;
            open = true;
        } else if (iv.first > hi) {
            busy += hi - lo;
            lo = iv.first;
            hi = iv.second;
        } else {
            hi = std::max(hi, iv.second);
        }
        last = std::max(last, iv.second);
    }
    if (open) busy += hi - lo;
    if (h2d_bytes) *h2d_bytes = h2d_bytes_;
    if (d2h_bytes) *d2h_bytes = d2h_bytes_;
    if (busy_ms) *busy_ms = busy;
    if (window_ms) *window_ms = open ? last - first : 0.0;
    if (scheduler_ms) *scheduler_ms = launch_ms_;
}

// Scheduler thread: reap finished batches, admit queued requests in order while the HBM budget
// holds them, launch them as one batch on a free stream. Called with mu_ held.
void Server::launch(std::vector<Request*>& reqs) {
    int s = -1;
    for (int i = 0; i < int(streams_.size()); ++i) {
        const int c = (next_stream_ + i) % int(streams_.size());
        if (!stream_busy_[size_t(c)]) {
            s = c;
            break;
        }
    }
    next_stream_ = (s + 1) % int(streams_.size());
    cudaStream_t st = streams_[size_t(s)];
    Batch& batch = *batches_[size_t(s)];
    batch.clear();
    // A request whose cached operand is gone (it cannot be: submit pins it and release_operand
    // refuses operands of queued requests) fails on its own instead of reading a null operand.
    std::vector<Request*> run;
    for (Request* r : reqs) {
        if (r->operand >= 0 && operands_.find(r->operand) == operands_.end()) {
            dev_arena_.free(r->dev);
            r->dev = nullptr;
            r->status = -1;
            continue;
        }
        run.push_back(r);
    }
    if (run.size() != reqs.size()) done_cv_.notify_all();
    reqs.swap(run);
    if (reqs.empty()) return;
    Flight f;
    try {
        check(cudaEventCreate(&f.begin), "event");
        check(cudaEventRecord(f.begin, st), "event");
        for (Request* r : reqs) {
            const size_t bytes = r->plan->limbs() * 4;
            char* da = r->dev;
            char* db = r->dev + r->limb_bytes;
            char* dc = r->dev + 2 * r->limb_bytes;
            uint64_t* scratch = reinterpret_cast<uint64_t*>(r->dev + 3 * r->limb_bytes);
            if (r->operand < 0) check(cudaMemcpyAsync(da, r->host, bytes, cudaMemcpyHostToDevice, st), "operand copy");
            check(cudaMemcpyAsync(db, r->host + r->limb_bytes, bytes, cudaMemcpyHostToDevice, st), "operand copy");
            f.h2d += bytes * (r->operand < 0 ? 2 : 1);
            f.d2h += bytes;
            if (r->operand >= 0)
                batch.add(r->plan, kModeCachedA, nullptr, reinterpret_cast<uint32_t*>(db),
                          reinterpret_cast<uint32_t*>(dc),
                          reinterpret_cast<const uint64_t*>(operands_.at(r->operand).dev), nullptr, scratch);
            else
                batch.add(r->plan, kModeProduct, reinterpret_cast<uint32_t*>(da), reinterpret_cast<uint32_t*>(db),
                          reinterpret_cast<uint32_t*>(dc), nullptr, nullptr, scratch);
            r->status = 1;
        }
        batch.run(st, false);
        for (Request* r : reqs)
            check(cudaMemcpyAsync(r->host + 2 * r->limb_bytes, r->dev + 2 * r->limb_bytes, r->plan->limbs() * 4,
                                  cudaMemcpyDeviceToHost, st),
                  "product copy");
        f.reqs = reqs;
        f.stream = s;
        check(cudaEventCreate(&f.done), "event");
        check(cudaEventRecord(f.done, st), "event");
    } catch (...) {
        // copies or kernels of this batch may already be queued: the caller frees the requests'
        // device blocks, so wait until nothing on the stream can still touch them
        cudaStreamSynchronize(st);
        if (f.begin) cudaEventDestroy(f.begin);
        if (f.done) cudaEventDestroy(f.done);
        throw;
    }
    stream_busy_[size_t(s)] = true;
    flights_.push_back(std::move(f));
    ++batches_run_;
}

bool Server::reap(bool) {
    bool any = false;
    for (auto it = flights_.begin(); it != flights_.end();) {
        const cudaError_t q = cudaEventQuery(it->done);
        if (q == cudaErrorNotReady) {
            ++it;
            continue;
        }
        const double t = now_ms();
        const bool timed_out = q == cudaSuccess && batches_[size_t(it->stream)]->failed();
        if (timed_out) {
            ++timeouts_;
            last_timeout_ = batches_[size_t(it->stream)]->failure();
        }
        for (Request* r : it->reqs) {
            dev_arena_.free(r->dev);
            r->dev = nullptr;
            if (timed_out) {
                r->status = -4;
            } else if (q == cudaSuccess) {
                r->status = 2;
                r->t_done = t;
                latencies_.push_back(t - r->t_submit);
                t_last_ = t;
            } else {
                r->status = -1;
            }
        }
        if (q != cudaSuccess) {
            fault_ = cudaGetErrorString(q);
        } else {
            float b = 0.f, e = 0.f;
            if (cudaEventElapsedTime(&b, origin_, it->begin) == cudaSuccess &&
                cudaEventElapsedTime(&e, origin_, it->done) == cudaSuccess)
                busy_.emplace_back(double(b), double(e));
            h2d_bytes_ += it->h2d;
            d2h_bytes_ += it->d2h;
        }
        cudaEventDestroy(it->begin);
        cudaEventDestroy(it->done);
        stream_busy_[size_t(it->stream)] = false;
        it = flights_.erase(it);
        any = true;
    }
    if (any) done_cv_.notify_all();
    return any;
}

void Server::loop() {
    if (cudaSetDevice(device_) != cudaSuccess) fault_ = "cannot select the server's device";
    std::unique_lock<std::mutex> lock(mu_);
    for (;;) {
        if (stop_ && queue_.empty() && flights_.empty()) return;
        reap(false);
        const bool free_stream = std::find(stream_busy_.begin(), stream_busy_.end(), false) != stream_busy_.end();
        std::vector<Request*> admit;
        if (free_stream && fault_.empty()) {
            while (!queue_.empty() && int(admit.size()) < max_batch_) {
                Request* r = queue_.front();
                r->dev = dev_arena_.alloc(r->dev_bytes);
                if (!r->dev) break;  // in order: wait for memory rather than let later requests pass
                queue_.pop_front();
                admit.push_back(r);
            }
        }
        if (!admit.empty()) {
            const double t_launch = now_ms();
            try {
                launch(admit);
                launch_ms_ += now_ms() - t_launch;
            } catch (const Error& e) {
                fault_ = e.what();
                for (Request* r : admit) {
                    dev_arena_.free(r->dev);
                    r->status = -1;
                }
                done_cv_.notify_all();
            }
            continue;
        }
        if (!fault_.empty()) {
            for (Request* r : queue_) r->status = -1;
            queue_.clear();
            done_cv_.notify_all();
        } else if (flights_.empty() && !queue_.empty()) {
            // nothing in flight will free memory: the head request cannot fit beside the
            // registered operands, so it fails instead of blocking the queue
            queue_.front()->status = -3;
            queue_.pop_front();
            done_cv_.notify_all();
            continue;
        }
        if (flights_.empty())
            cv_.wait(lock, [&] { return stop_ || !queue_.empty(); });
        else
            cv_.wait_for(lock, std::chrono::microseconds(20));
    }
}

}  // namespace nc
