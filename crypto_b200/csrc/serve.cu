// Served KZG commits: a request loop over the resident SRS with continuous
// batching.
//
// Requests (evaluations of one polynomial each) are queued by submitters.
// One worker thread owns `slots` execution slots, each with its own CUDA
// stream and CommitBatcher.  Whenever a slot is idle and requests are
// waiting, the worker forms a batch from the head of the queue (up to
// max_batch requests), admitting requests one by one while the batch's
// computed device footprint (evaluations, NTT scratch, MSM buckets and
// entries) fits the memory budget and the device's free memory, and queues
// it on that slot.  Batches on different slots overlap on the device; a
// request that arrives while others are running is admitted as soon as a
// slot frees.  Completion is detected with events, results are copied to
// pinned memory, and each request records submit-to-completion latency.
// Every commit is exact, so a request's result is the same bytes alone or
// in any mix.
#include "../../include/kinet_b200/crypto_b200.h"
#include "batch.cuh"
#include "kzg.cuh"
#include "runtime.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <set>
#include <mutex>
#include <thread>
#include <vector>

namespace kb200 {

// Resident SRS of the calling thread's device (owned by the C-ABI context).
void resident_srs(const uint32_t** table, size_t* n);
ShiftTables* resident_srs_shifts();

namespace {

using Clock = std::chrono::steady_clock;

// Pinned host slabs for request payloads, recycled by power-of-two size
// class: a request is copied once, at submit, into page-locked memory, and
// its batch's host-to-device copy reads it from there asynchronously.
// Slabs are carved from one arena pinned at server creation: page-locking
// under load (cudaHostAlloc, tens of ms for a few MiB) holds a driver lock
// that stalls the worker's launches.  An exhausted arena falls back to
// cudaHostAlloc.
class PinnedPool {
   public:
    ~PinnedPool() {
        for (void* p : all_) cudaFreeHost(p);
        if (base_) cudaFreeHost(base_);
    }
    void reserve_arena(size_t bytes) {
        KB_CUDA(cudaHostAlloc(&base_, bytes, cudaHostAllocPortable));
        cap_ = bytes;
    }
    static size_t size_class(size_t bytes) {
        size_t c = 4096;
        while (c < bytes) c <<= 1;
        return c;
    }
    uint8_t* get(size_t bytes) {
        const size_t c = size_class(bytes);
        {
            std::lock_guard<std::mutex> lk(mu_);
            auto& v = free_[c];
            if (!v.empty()) {
                void* p = v.back();
                v.pop_back();
                return static_cast<uint8_t*>(p);
            }
            if (base_ && used_ + c <= cap_) {
                uint8_t* p = static_cast<uint8_t*>(base_) + used_;
                used_ += c;
                return p;
            }
        }
        void* p = nullptr;
        const auto t0 = Clock::now();
        KB_CUDA(cudaHostAlloc(&p, c, cudaHostAllocPortable));
        if (alloc_trace_enabled())
            std::fprintf(stderr, "[pinned] %zu bytes, %.3f ms\n", c,
                         std::chrono::duration<double, std::milli>(Clock::now() - t0).count());
        std::lock_guard<std::mutex> lk(mu_);
        all_.push_back(p);
        return static_cast<uint8_t*>(p);
    }
    void put(uint8_t* p, size_t bytes) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu_);
        free_[size_class(bytes)].push_back(p);
    }

   private:
    std::mutex mu_;
    std::map<size_t, std::vector<void*>> free_;
    std::vector<void*> all_;
    void* base_ = nullptr;
    size_t cap_ = 0, used_ = 0;
};

struct Request {
    uint64_t ticket = 0;
    uint8_t* evals = nullptr;  // pinned slab of n * 32 bytes (returned at completion)
    size_t n = 0;
    uint8_t commit[48] = {};
    int status = 1;  // 1 pending, 0 done, < 0 error
    Clock::time_point t_submit, t_done;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    CommitBatcher* batcher = nullptr;
    HostBuf h_out;
    std::vector<Request*> reqs;
    bool busy = false;
    std::chrono::steady_clock::time_point t_launch;
};

}  // namespace

class KzgServer {
   public:
    int device = 0;
    size_t max_batch = 64;
    size_t mem_budget = 0;
    const uint32_t* srs = nullptr;
    size_t srs_n = 0;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::map<uint64_t, Request*> by_ticket;
    std::vector<double> latencies_ms;
    PinnedPool pool;
    uint64_t next_ticket = 1;
    uint64_t completed = 0;
    Clock::time_point first_submit, last_done;
    bool have_first = false;
    std::atomic<bool> stop{false};
    bool trace = std::getenv("KB200_SERVE_TRACE") != nullptr;  // per-batch log on stderr
    std::string error;
    std::thread worker;

    // Free device memory for admission.  cudaMemGetInfo is queried only while
    // no batch of this server is in flight, at most once a second: measured
    // on B200, calls made while large kernels ran stalled the worker thread
    // for tens of milliseconds, which showed up as p99 latency.
    size_t free_snapshot = 0;
    Clock::time_point free_at{};
    size_t device_free() {
        bool busy = false;
        for (const Slot& sl : slots) busy |= sl.busy;
        const auto now = Clock::now();
        if (free_snapshot == 0 || (!busy && now - free_at > std::chrono::seconds(1))) {
            size_t f = 0, t = 0;
            if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
                cudaGetLastError();
                f = 0;
            }
            free_snapshot = f;
            free_at = now;
        }
        return free_snapshot;
    }
    void loop();
    bool launch_batch(Slot& s);
    void finish(Slot& s);
};

void KzgServer::finish(Slot& s) {
    const auto now = Clock::now();
    if (trace)
        std::fprintf(stderr, "[kzg_server] slot %d: done after %.3f ms\n", (int)(&s - slots.data()),
                     std::chrono::duration<double, std::milli>(now - s.t_launch).count());
    std::lock_guard<std::mutex> lk(mu);
    for (size_t i = 0; i < s.reqs.size(); ++i) {
        Request* r = s.reqs[i];
        std::memcpy(r->commit, s.h_out.as<uint8_t>() + 48 * i, 48);
        pool.put(r->evals, r->n * 32);
        r->evals = nullptr;
        r->t_done = now;
        r->status = 0;
        latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
        ++completed;
    }
    last_done = now;
    s.reqs.clear();
    s.busy = false;
    cv_done.notify_all();
}

bool KzgServer::launch_batch(Slot& s) {
    std::vector<Request*> take;
    std::vector<size_t> sizes;
    {
        std::lock_guard<std::mutex> lk(mu);
        const size_t free_b = device_free();
        const size_t headroom = (size_t)256 << 20;
        const size_t avail = free_b > headroom ? free_b - headroom : 0;
        const size_t cap = mem_budget ? std::min(mem_budget, avail + 0) : avail;
        size_t need = commit_batch_fixed_bytes();
        while (!queue.empty() && take.size() < max_batch) {
            Request* r = queue.front();
            const size_t item = commit_item_scratch_bytes(r->n);
            // Admit at least one request when the device is otherwise idle, so
            // a single oversized request is attempted rather than starved.
            if (need + item > cap && !take.empty()) break;
            need += item;
            sizes.push_back(r->n);
            take.push_back(r);
            queue.pop_front();
        }
    }
    if (take.empty()) return false;
    const auto t_launch = Clock::now();
    size_t total = 0;
    for (Request* r : take) total += r->n;
    if (s.h_out.bytes < take.size() * 48) s.h_out.reserve(std::max<size_t>(max_batch, take.size()) * 48, s.stream);
    uint8_t* d_in = commit_batch_device_input(s.batcher, sizes.data(), sizes.size(), srs, srs_n,
                                              s.stream);
    const auto t_prep = Clock::now();
    size_t off = 0;
    for (Request* r : take) {
        KB_CUDA(cudaMemcpyAsync(d_in + off * 32, r->evals, r->n * 32, cudaMemcpyHostToDevice,
                                s.stream));
        off += r->n;
    }
    const auto t_copy = Clock::now();
    commit_batch_device(s.batcher, sizes.data(), sizes.size(), srs, srs_n, s.stream,
                        /*use_graph=*/false);
    KB_CUDA(cudaMemcpyAsync(s.h_out.ptr, commit_batch_device_output(s.batcher), take.size() * 48,
                            cudaMemcpyDeviceToHost, s.stream));
    KB_CUDA(cudaEventRecord(s.done, s.stream));
    if (trace) {
        const size_t free_b = free_snapshot;
        using ms = std::chrono::duration<double, std::milli>;
        std::fprintf(stderr, "[kzg_server] slot %d: %zu requests (%zu evaluations), host %.3f ms "
                             "(prepare %.3f, copies %.3f), queue left %zu, free %.1f GB\n",
                     (int)(&s - slots.data()), take.size(), total, ms(Clock::now() - t_launch).count(),
                     ms(t_prep - t_launch).count(), ms(t_copy - t_prep).count(), queue.size(),
                     free_b / 1e9);
    }
    s.reqs = std::move(take);
    s.busy = true;
    s.t_launch = t_launch;
    return true;
}

void KzgServer::loop() {
    // Buffers that grow under load keep their old allocations (a free waits
    // for the other slot's batch, and at times far longer); they are freed
    // while both slots are idle once they pass 1 GiB, and at exit.
    devbuf_defer_frees(true);
    try {
        KB_CUDA(cudaSetDevice(device));
        while (!stop.load()) {
            bool progressed = false;
            for (Slot& s : slots) {
                if (s.busy) {
                    const cudaError_t q = cudaEventQuery(s.done);
                    if (q == cudaSuccess) {
                        finish(s);
                        progressed = true;
                    } else if (q != cudaErrorNotReady) {
                        KB_CUDA(q);
                    }
                }
            }
            for (Slot& s : slots) {
                if (!s.busy && launch_batch(s)) progressed = true;
            }
            if (!progressed) {
                bool idle = true;
                for (Slot& s : slots) idle &= !s.busy;
                if (idle && devbuf_retired_bytes() > ((size_t)1 << 30)) devbuf_free_retired();
                std::unique_lock<std::mutex> lk(mu);
                bool any_busy = false;
                for (Slot& s : slots) any_busy |= s.busy;
                if (any_busy)
                    cv_work.wait_for(lk, std::chrono::microseconds(50));
                else
                    cv_work.wait_for(lk, std::chrono::milliseconds(2),
                                     [&] { return stop.load() || !queue.empty(); });
            }
        }
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(mu);
        error = e.what();
        for (auto& kv : by_ticket)
            if (kv.second->status == 1) kv.second->status = KB200_CRYPTO_ERR_BACKEND;
        cv_done.notify_all();
    }
    for (Slot& s : slots) cudaStreamSynchronize(s.stream);
    devbuf_free_retired();
}

}  // namespace kb200

using namespace kb200;

extern "C" {

void* kzg_server_create(size_t max_batch, int slots, size_t mem_budget_bytes) {
    try {
        auto* s = new KzgServer();
        KB_CUDA(cudaGetDevice(&s->device));
        resident_srs(&s->srs, &s->srs_n);
        if (!s->srs || !s->srs_n) {
            set_last_error("kzg_server_create: no resident SRS (load or generate one first)");
            delete s;
            return nullptr;
        }
        s->max_batch = max_batch ? max_batch : 64;
        s->mem_budget = mem_budget_bytes;
        {
            // Room for eight full-size requests in flight (or many smaller
            // ones); KB200_SERVE_PINNED_MB overrides.
            size_t arena = (size_t)8 * s->srs_n * 32;
            if (const char* v = std::getenv("KB200_SERVE_PINNED_MB"))
                if (*v) arena = (size_t)std::strtoull(v, nullptr, 10) << 20;
            if (arena) s->pool.reserve_arena(arena);
        }
        s->slots.resize(slots > 0 ? (size_t)slots : 2);
        for (Slot& sl : s->slots) {
            KB_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
            KB_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
            sl.batcher = commit_batcher_create();
            commit_batcher_set_shift(sl.batcher, resident_srs_shifts());
            commit_batcher_set_transient(sl.batcher, true);
        }
        // Build the shifted SRS tables every commit size can select now, so
        // no request pays for a table build.
        if (ShiftTables* sh = resident_srs_shifts()) {
            std::set<int> cs;
            for (size_t n = 1; n <= s->srs_n; n <<= 1) cs.insert(shift_c_for(&n, 1));
            for (int c : cs) shift_tables_get(sh, c, s->slots[0].stream);
        }
        // Warm every slot with the largest batches it is likely to see, so
        // its engines, plans and staging reach their working size before the
        // first request instead of growing under load (an allocation there
        // waits on the device and, on a busy device, at times for hundreds
        // of milliseconds): a full-SRS commit plus max_batch - 1 commits of up
        // to 2^16, and for every window-size class the batcher groups commits
        // by, max_batch commits of the class's largest size (at most 2^22
        // evaluations in all).
        {
            std::vector<std::vector<size_t>> shapes;
            {
                std::vector<size_t> mixed{s->srs_n};
                const size_t mid = std::min<size_t>(s->srs_n, (size_t)1 << 16);
                for (size_t k = 1; k < s->max_batch; ++k) mixed.push_back(mid);
                shapes.push_back(mixed);
            }
            std::map<int, size_t> largest;  // window class -> largest size in it
            for (size_t n = 1; n <= s->srs_n; n <<= 1) largest[shift_c_for(&n, 1)] = n;
            for (const auto& kv : largest) {
                const size_t n = kv.second;
                const size_t cnt = std::max<size_t>(1, std::min(s->max_batch, ((size_t)1 << 22) / n));
                shapes.push_back(std::vector<size_t>(cnt, n));
            }
            for (const auto& sizes : shapes) {
                size_t total = 0;
                for (size_t v : sizes) total += v;
                for (Slot& sl : s->slots) {
                    uint8_t* d_in = commit_batch_device_input(sl.batcher, sizes.data(), sizes.size(),
                                                              s->srs, s->srs_n, sl.stream);
                    KB_CUDA(cudaMemsetAsync(d_in, 0, total * 32, sl.stream));
                    commit_batch_device(sl.batcher, sizes.data(), sizes.size(), s->srs, s->srs_n,
                                        sl.stream, /*use_graph=*/false);
                    KB_CUDA(cudaStreamSynchronize(sl.stream));
                }
            }
            for (Slot& sl : s->slots) sl.h_out.reserve(s->max_batch * 48, sl.stream);
        }
        s->device_free();  // first admission snapshot, device idle after the warm-up
        s->worker = std::thread([s] { s->loop(); });
        return s;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return nullptr;
    }
}

int kzg_server_submit(void* handle, const uint8_t* evals32le, size_t n, uint64_t* ticket) {
    auto* s = static_cast<KzgServer*>(handle);
    if (!s || !evals32le || !ticket) return KB200_CRYPTO_ERR_INPUT;
    if (n == 0 || (n & (n - 1))) return KB200_CRYPTO_ERR_LENGTH;
    if (n > s->srs_n) return KB200_CRYPTO_ERR_LENGTH;
    auto* r = new Request();
    try {
        r->evals = s->pool.get(n * 32);
    } catch (const std::exception& e) {
        delete r;
        set_last_error(e.what());
        return KB200_CRYPTO_ERR_BACKEND;
    }
    std::memcpy(r->evals, evals32le, n * 32);
    r->n = n;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->error.empty()) {
            s->pool.put(r->evals, n * 32);
            delete r;
            set_last_error(s->error);
            return KB200_CRYPTO_ERR_BACKEND;
        }
        r->ticket = s->next_ticket++;
        if (!s->have_first) {
            s->first_submit = r->t_submit;
            s->have_first = true;
        }
        s->by_ticket[r->ticket] = r;
        s->queue.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return KB200_CRYPTO_OK;
}

// Blocks until the request completes (timeout_ms < 0: no limit).  Returns 0
// with the commitment, 1 on timeout, or a negative error.  The ticket is
// released on completion.
int kzg_server_wait(void* handle, uint64_t ticket, uint8_t commit48[48], double* latency_ms,
                    double timeout_ms) {
    auto* s = static_cast<KzgServer*>(handle);
    if (!s || !commit48) return KB200_CRYPTO_ERR_INPUT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->by_ticket.find(ticket);
    if (it == s->by_ticket.end()) return KB200_CRYPTO_ERR_INPUT;
    Request* r = it->second;
    auto pred = [&] { return r->status != 1; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred))
        return 1;
    const int st = r->status;
    if (st == 0) {
        std::memcpy(commit48, r->commit, 48);
        if (latency_ms)
            *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    } else {
        set_last_error(s->error);
    }
    s->by_ticket.erase(it);
    delete r;
    return st;
}

// Latency percentiles over completed requests since creation or the last
// reset, sustained commits/s from the first submit to the last completion.
int kzg_server_stats(void* handle, double* p50_ms, double* p99_ms, double* commits_per_s,
                     uint64_t* completed, int reset) {
    auto* s = static_cast<KzgServer*>(handle);
    if (!s) return KB200_CRYPTO_ERR_INPUT;
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> v = s->latencies_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {
        if (v.empty()) return 0.0;
        size_t k = (size_t)(q * (double)(v.size() - 1) + 0.5);
        return v[std::min(k, v.size() - 1)];
    };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (completed) *completed = s->completed;
    if (commits_per_s) {
        const double secs =
            s->have_first ? std::chrono::duration<double>(s->last_done - s->first_submit).count() : 0;
        *commits_per_s = secs > 0 ? (double)s->completed / secs : 0.0;
    }
    if (reset) {
        s->latencies_ms.clear();
        s->completed = 0;
        s->have_first = false;
    }
    return KB200_CRYPTO_OK;
}

int kzg_server_destroy(void* handle) {
    auto* s = static_cast<KzgServer*>(handle);
    if (!s) return KB200_CRYPTO_ERR_INPUT;
    s->stop.store(true);
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (Slot& sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        commit_batcher_destroy(sl.batcher);
        sl.h_out.release();
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    for (auto& kv : s->by_ticket) delete kv.second;
    delete s;
    return KB200_CRYPTO_OK;
}

}  // extern "C"
