// Batched KZG commits: see batch.cuh.
#include "batch.cuh"
#include "kzg.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>

namespace kb200 {

namespace {

struct Signature {
    std::vector<size_t> sizes;
    const uint32_t* srs;
    uint64_t shift_gen;  // shifted-table generation (0 = none)
    bool operator<(const Signature& o) const {
        if (srs != o.srs) return srs < o.srs;
        if (shift_gen != o.shift_gen) return shift_gen < o.shift_gen;
        return sizes < o.sizes;
    }
};

struct MsmGroup {
    MsmBatchPlan* plan = nullptr;
    const uint32_t* table = nullptr;  // SRS, or its shifted levels for the group's window size
};

struct Prepared {
    std::vector<MsmGroup> groups;                    // the first ngroups are in use
    size_t ngroups = 0;
    std::vector<std::pair<size_t, size_t>> classes;  // (n, count) per size class
    std::vector<size_t> class_off;                   // start in the offsets list
    DevBuf d_vec_off;                                // element offsets grouped by class
    size_t total = 0;                                // evaluations
    cudaGraphExec_t graph = nullptr;
    unsigned long long graph_moves = 0;  // devbuf_moves() when the graph was captured
    ~Prepared() {
        if (graph) cudaGraphExecDestroy(graph);
        for (MsmGroup& g : groups) msm_batch_plan_destroy(g.plan);
        d_vec_off.release();
    }
};

}  // namespace

class CommitBatcher {
   public:
    NttEngine* ntt = nullptr;
    MsmEngine* msm = nullptr;
    DevBuf evals, scratch, out_wire, out_comp;
    HostBuf h_out;
    std::map<Signature, std::unique_ptr<Prepared>> cache;
    Prepared* current = nullptr;
    ShiftTables* shifts = nullptr;
    // Transient mode (serving, where batch signatures rarely repeat): one
    // Prepared is rebuilt in place for every batch, reusing its device
    // buffers, instead of caching (and later freeing) one per signature.
    bool transient = false;
    std::unique_ptr<Prepared> scratch_prep;
    std::vector<size_t> scratch_sizes;  // sizes scratch_prep was last built for
    unsigned long long graph_launches = 0, graph_captures = 0;
    ~CommitBatcher() {
        cache.clear();
        if (ntt) ntt_engine_destroy(ntt);
        if (msm) msm_engine_destroy(msm);
        for (DevBuf* b : {&evals, &scratch, &out_wire, &out_comp}) b->release();
        h_out.release();
    }
};

CommitBatcher* commit_batcher_create() {
    auto* b = new CommitBatcher();
    b->ntt = ntt_engine_create(2);
    b->msm = msm_engine_create(2);
    return b;
}

void commit_batcher_destroy(CommitBatcher* b) { delete b; }

void commit_batcher_set_shift(CommitBatcher* b, ShiftTables* shifts) { b->shifts = shifts; }
void commit_batcher_set_transient(CommitBatcher* b, bool transient) { b->transient = transient; }

static Prepared* prepare(CommitBatcher* B, const size_t* sizes, size_t count,
                         const uint32_t* srs, size_t srs_n, cudaStream_t st) {
    const bool shifted = B->shifts && shift_tables_stride(B->shifts) == srs_n;
    Signature sig{std::vector<size_t>(sizes, sizes + count), srs,
                  shifted ? shift_tables_generation(B->shifts) : 0};
    std::unique_ptr<Prepared> fresh;
    Prepared* P;
    if (B->transient) {
        if (!B->scratch_prep) B->scratch_prep = std::make_unique<Prepared>();
        P = B->scratch_prep.get();
        // commit_batch_device_input and commit_batch_device prepare the same
        // batch back to back: build it once
        if (P->ngroups && B->scratch_sizes == sig.sizes) return P;
        B->scratch_sizes = sig.sizes;
        P->classes.clear();
        P->class_off.clear();
    } else {
        auto it = B->cache.find(sig);
        if (it != B->cache.end()) return it->second.get();
        fresh = std::make_unique<Prepared>();
        P = fresh.get();
    }
    std::vector<MsmItem> items(count);
    std::map<size_t, std::vector<unsigned long long>> by_size;
    size_t off = 0;
    for (size_t i = 0; i < count; ++i) {
        const size_t n = sizes[i];
        if (n == 0 || (n & (n - 1))) throw std::invalid_argument("kzg: sizes must be powers of two");
        if (n > srs_n) throw std::invalid_argument("kzg: SRS shorter than the polynomial");
        items[i] = MsmItem{off, n, 0};
        by_size[n].push_back(off);
        off += n;
    }
    P->total = off;
    std::vector<unsigned long long> offs;
    for (auto& kv : by_size) {
        P->class_off.push_back(offs.size());
        P->classes.emplace_back(kv.first, kv.second.size());
        offs.insert(offs.end(), kv.second.begin(), kv.second.end());
        ntt_prepare(B->ntt, kv.first, 0, st);
    }
    P->d_vec_off.reserve(std::max<size_t>(1, offs.size()) * 8, st);
    if (!offs.empty())
        KB_CUDA(cudaMemcpyAsync(P->d_vec_off.ptr, offs.data(), offs.size() * 8,
                                cudaMemcpyHostToDevice, st));
    // MSM groups: against shifted tables every commit joins the group of its
    // own best window size (results go to its slot through out_index), so a
    // large commit does not impose its window on the small ones; otherwise
    // one plain plan for the whole batch.
    std::map<int, std::vector<MsmItem>> by_c;
    for (size_t i = 0; i < count; ++i) {
        MsmItem it = items[i];
        it.out_index = i;
        by_c[shifted ? shift_c_for(&sizes[i], 1) : 0].push_back(it);
    }
    P->ngroups = 0;
    for (auto& kv : by_c) {
        MsmOptions opt;
        const uint32_t* table = srs;
        if (kv.first > 0) {
            if (const uint32_t* t = shift_tables_get(B->shifts, kv.first, st)) {
                opt.shift_c = kv.first;
                opt.shift_stride = srs_n;
                table = t;
            }
        }
        if (P->ngroups < P->groups.size()) {
            MsmGroup& g = P->groups[P->ngroups];
            msm_batch_plan_update(g.plan, kv.second.data(), kv.second.size(), opt, st);
            g.table = table;
        } else {
            MsmGroup g;
            g.table = table;
            g.plan = msm_batch_plan_create(2, kv.second.data(), kv.second.size(), opt, st);
            P->groups.push_back(g);
        }
        msm_engine_reserve(B->msm, P->groups[P->ngroups].plan, st);
        ++P->ngroups;
    }
    B->evals.reserve(std::max<size_t>(1, off) * 32 + 16, st);
    B->scratch.reserve(std::max<size_t>(1, off) * 32 + 16, st);
    B->out_wire.reserve(std::max<size_t>(1, count) * 96, st);
    B->out_comp.reserve(std::max<size_t>(1, count) * 48, st);
    B->h_out.reserve(std::max<size_t>(1, count) * 48, st);
    if (B->transient) return P;
    KB_CUDA(cudaStreamSynchronize(st));
    Prepared* raw = fresh.get();
    B->cache[sig] = std::move(fresh);
    if (B->cache.size() > 32) {
        // Bound the cache; keep the current signature.
        for (auto i2 = B->cache.begin(); i2 != B->cache.end();) {
            if (i2->second.get() != raw)
                i2 = B->cache.erase(i2);
            else
                ++i2;
        }
    }
    return raw;
}

// The device work of one batch: grouped inverse NTTs then the batched MSM.
static void enqueue(CommitBatcher* B, Prepared* P, const uint32_t* srs, cudaStream_t st) {
    static const bool trace = std::getenv("KB200_SERVE_TRACE") != nullptr;
    using Clk = std::chrono::steady_clock;
    auto t0 = Clk::now();
    auto lap = [&](const char* what, size_t arg) {
        if (!trace) return;
        const auto t1 = Clk::now();
        const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        if (ms > 2.0) std::fprintf(stderr, "[batcher] enqueue %s (%zu): %.3f ms\n", what, arg, ms);
        t0 = t1;
    };
    for (size_t k = 0; k < P->classes.size(); ++k) {
        const size_t n = P->classes[k].first, cnt = P->classes[k].second;
        ntt_run_list(B->ntt, B->evals.as<uint32_t>(), n, /*inverse=*/1, /*coset=*/0, cnt,
                     P->d_vec_off.as<unsigned long long>() + P->class_off[k],
                     B->scratch.as<uint32_t>(), st);
        lap("ntt", n);
    }
    (void)srs;
    for (size_t k = 0; k < P->ngroups; ++k) {
        msm_engine_launch(B->msm, P->groups[k].plan, B->evals.as<uint8_t>(), P->groups[k].table,
                          B->out_wire.as<uint8_t>(), B->out_comp.as<uint8_t>(), st);
        lap("msm group", k);
    }
}

static void run(CommitBatcher* B, Prepared* P, const uint32_t* srs, cudaStream_t st,
                bool use_graph) {
    if (!use_graph || B->transient) {
        enqueue(B, P, srs, st);
        return;
    }
    if (P->graph && P->graph_moves != devbuf_moves()) {
        // a buffer the graph addresses may have moved since the capture
        // (another batch shape grew the engine): capture again
        cudaGraphExecDestroy(P->graph);
        P->graph = nullptr;
    }
    if (!P->graph) {
        cudaGraph_t g = nullptr;
        KB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue(B, P, srs, st);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        KB_CUDA(cudaStreamEndCapture(st, &g));
        const cudaError_t err = cudaGraphInstantiate(&P->graph, g, 0);
        cudaGraphDestroy(g);
        KB_CUDA(err);
        P->graph_moves = devbuf_moves();
        ++B->graph_captures;
    }
    KB_CUDA(cudaGraphLaunch(P->graph, st));
    ++B->graph_launches;
}

void commit_batch_host(CommitBatcher* B, const uint8_t* h_evals, const size_t* sizes,
                       size_t count, const uint32_t* srs, size_t srs_n, uint8_t* h_out,
                       cudaStream_t st, bool use_graph) {
    if (count == 0) return;
    Prepared* P = prepare(B, sizes, count, srs, srs_n, st);
    B->current = P;
    KB_CUDA(cudaMemcpyAsync(B->evals.ptr, h_evals, P->total * 32, cudaMemcpyHostToDevice, st));
    run(B, P, srs, st, use_graph);
    KB_CUDA(cudaMemcpyAsync(B->h_out.ptr, B->out_comp.ptr, count * 48, cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    std::memcpy(h_out, B->h_out.ptr, count * 48);
}

uint8_t* commit_batch_device_input(CommitBatcher* B, const size_t* sizes, size_t count,
                                   const uint32_t* srs, size_t srs_n, cudaStream_t st) {
    Prepared* P = prepare(B, sizes, count, srs, srs_n, st);
    B->current = P;
    return B->evals.as<uint8_t>();
}

void commit_batch_device(CommitBatcher* B, const size_t* sizes, size_t count,
                         const uint32_t* srs, size_t srs_n, cudaStream_t st, bool use_graph) {
    if (count == 0) return;
    Prepared* P = prepare(B, sizes, count, srs, srs_n, st);
    B->current = P;
    run(B, P, srs, st, use_graph);
}

const uint8_t* commit_batch_device_output(CommitBatcher* B) { return B->out_comp.as<uint8_t>(); }

size_t commit_item_scratch_bytes(size_t n) { return 2 * n * 32 + 144 + msm_item_scratch_bytes(2, n); }
size_t commit_batch_fixed_bytes() { return msm_batch_fixed_bytes(2); }

size_t commit_batch_scratch_bytes(const size_t* sizes, size_t count) {
    size_t b = commit_batch_fixed_bytes();
    for (size_t i = 0; i < count; ++i) b += commit_item_scratch_bytes(sizes[i]);
    return b;
}

unsigned long long commit_batcher_graph_launches(CommitBatcher* b) { return b->graph_launches; }
unsigned long long commit_batcher_graph_captures(CommitBatcher* b) { return b->graph_captures; }

}  // namespace kb200
