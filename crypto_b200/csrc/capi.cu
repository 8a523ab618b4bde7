// C ABI: host-side glue between the reference-shaped entry points and the
// device engines.  Per device there is one context (stream, engines, I/O
// staging, resident SRS) guarded by a mutex.
#include "../../include/kinet_b200/crypto_b200.h"
#include "batch.cuh"
#include "eip2537.cuh"
#include "curve.cuh"
#include "kzg.cuh"
#include "kzg_blob.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "runtime.cuh"
#include "wntt.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>

namespace kb200 {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<unsigned long long> g_launches{0};
static std::atomic<bool> g_profile{false};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
bool profiling_enabled() { return g_profile.load(std::memory_order_relaxed); }

bool alloc_trace_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("KB200_ALLOC_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}

void alloc_trace(size_t from, size_t to, double ms) {
    std::fprintf(stderr, "[devbuf] %zu -> %zu bytes, %.3f ms\n", from, to, ms);
}

struct DeviceCtx {
    int dev = -1;
    std::mutex mu;
    cudaStream_t stream = nullptr;
    MsmEngine* msm[3] = {nullptr, nullptr, nullptr};
    NttEngine* ntt[3] = {nullptr, nullptr, nullptr};
    FixedBase* fb[3] = {nullptr, nullptr, nullptr};
    CommitBatcher* batcher = nullptr;
    WordNttCache* wntt = nullptr;
    ShiftTables* srs_shift = nullptr;  // shifted levels of d_srs
    ShiftTables* srs_shift_get() {
        if (!srs_shift) srs_shift = shift_tables_create();
        return srs_shift;
    }
    BlobSetup* blob = nullptr;
    DevBuf d_bl;  // blob ops: input, z, outputs, flag
    BlobSetup* blob_get() {
        if (!blob) blob = blob_setup_create();
        return blob;
    }
    DevBuf d_a, d_b, d_out, d_srs, d_tmp, d_w, d_ws, d_e_in, d_e_tab, d_e_sc, d_e_out;
    HostBuf h_a, h_b, h_out;
    size_t srs_n = 0;

    MsmEngine* msm_for(int curve) {
        if (!msm[curve]) msm[curve] = msm_engine_create(curve);
        return msm[curve];
    }
    NttEngine* ntt_for(int curve) {
        if (!ntt[curve]) ntt[curve] = ntt_engine_create(curve);
        return ntt[curve];
    }
    FixedBase* fb_for(int curve) {
        if (!fb[curve]) fb[curve] = fixed_base_create(curve, stream);
        return fb[curve];
    }
    WordNttCache* wntt_get() {
        if (!wntt) wntt = word_ntt_cache_create();
        return wntt;
    }
    CommitBatcher* batcher_get() {
        if (!batcher) {
            batcher = commit_batcher_create();
            commit_batcher_set_shift(batcher, srs_shift_get());
        }
        return batcher;
    }
};

static std::mutex g_ctx_mu;
static std::map<int, std::unique_ptr<DeviceCtx>> g_ctx;

static DeviceCtx* get_ctx() {
    int count = 0;
    cudaError_t err = cudaGetDeviceCount(&count);
    if (err != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw CudaError(err == cudaSuccess ? cudaErrorNoDevice : err,
                        "no usable CUDA device (kinet-b200 has no CPU fallback)");
    }
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto& slot = g_ctx[dev];
    if (!slot) {
        auto c = std::make_unique<DeviceCtx>();
        c->dev = dev;
        KB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        slot = std::move(c);
    }
    return slot.get();
}

// Runs fn, mapping exceptions to the given error codes.
template <class Fn>
static int guarded(int backend_err, int size_err, int internal_err, Fn&& fn) {
    try {
        return fn();
    } catch (const CudaError& e) {
        set_last_error(e.what());
        return backend_err;
    } catch (const std::invalid_argument& e) {
        set_last_error(e.what());
        return size_err;
    } catch (const std::bad_alloc& e) {
        set_last_error("host allocation failed");
        return internal_err;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return internal_err;
    }
}

ShiftTables* resident_srs_shifts() {
    DeviceCtx* c = get_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    return c->srs_shift_get();
}

void resident_srs(const uint32_t** table, size_t* n) {
    DeviceCtx* c = get_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    *table = c->srs_n ? c->d_srs.as<uint32_t>() : nullptr;
    *n = c->srs_n;
}

static int wire_bytes(uint32_t curve) { return curve == 2 ? 96 : 64; }

static bool is_pow2(size_t n) { return n && !(n & (n - 1)); }

// ---- MSM -------------------------------------------------------------------

static int msm_host(uint32_t curve, const uint8_t* scalars, const uint8_t* points, size_t n,
                    uint8_t* result, bool points_in_g1) {
    if (!result) return KB200_GPUKIT_ERR_NULL_ARG;
    if (n > 0 && (!scalars || !points)) return KB200_GPUKIT_ERR_NULL_ARG;
    if (curve == 0 || curve == 3) {
        set_last_error("curve has no GPU body in kinet-b200 (secp256k1 / banderwagon)");
        return KB200_GPUKIT_ERR_NOTIMPL;
    }
    if (curve != 1 && curve != 2) return KB200_GPUKIT_ERR_BACKEND;
    return guarded(KB200_GPUKIT_ERR_DISPATCH, KB200_GPUKIT_ERR_BAD_SIZE, KB200_GPUKIT_ERR_DISPATCH,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       const size_t pb = (size_t)wire_bytes(curve);
                       cudaStream_t st = c->stream;
                       c->d_a.reserve(n * 32 + 16, st);
                       c->d_b.reserve(n * pb + 16, st);
                       c->d_out.reserve(256, st);
                       c->h_out.reserve(256, st);
                       MsmOptions opt;
                       opt.ref_carry_quirk = true;
                       opt.points_in_g1 = points_in_g1;
                       if (n) {
                           msm_run_host_wire(c->msm_for((int)curve), scalars, points, n,
                                             c->d_a.as<uint8_t>(), c->d_b.as<uint8_t>(),
                                             c->d_out.as<uint8_t>(), st, opt);
                       } else {
                           msm_run_wire(c->msm_for((int)curve), c->d_a.as<uint8_t>(),
                                        c->d_b.as<uint8_t>(), n, c->d_out.as<uint8_t>(), nullptr,
                                        st, opt);
                       }
                       KB_CUDA(cudaMemcpyAsync(c->h_out.ptr, c->d_out.ptr, pb,
                                               cudaMemcpyDeviceToHost, st));
                       KB_CUDA(cudaStreamSynchronize(st));
                       std::memcpy(result, c->h_out.ptr, pb);
                       return KB200_GPUKIT_OK;
                   });
}

// ---- NTT -------------------------------------------------------------------

static int ntt_host(int curve, uint8_t* data, size_t n, int inverse, int coset) {
    if (!data) return KB200_CRYPTO_ERR_INPUT;
    if (curve != 1 && curve != 2) return KB200_CRYPTO_ERR_INPUT;
    if (!is_pow2(n) || n > ((size_t)1 << ntt_max_log(curve))) return KB200_CRYPTO_ERR_LENGTH;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       cudaStream_t st = c->stream;
                       c->d_a.reserve(n * 32 + 16, st);
                       KB_CUDA(cudaMemcpyAsync(c->d_a.ptr, data, n * 32, cudaMemcpyHostToDevice, st));
                       ntt_run(c->ntt_for(curve), c->d_a.as<uint32_t>(), n, inverse, coset, 1, st);
                       KB_CUDA(cudaMemcpyAsync(data, c->d_a.ptr, n * 32, cudaMemcpyDeviceToHost, st));
                       KB_CUDA(cudaStreamSynchronize(st));
                       return KB200_CRYPTO_OK;
                   });
}

// ---- word-prime NTT -----------------------------------------------------------

// ntt_forward / ntt_inverse (ntt/c-abi/c_ntt.cpp:81-179): argument checks in
// the reference's order, then the transform on the device.  Invalid
// arguments return CRYPTO_ERR_INPUT before any data moves.
static bool word_ntt_args_ok(const uint64_t* coeffs, size_t n, uint64_t modulus) {
    if (!coeffs || !is_pow2(n)) return false;
    if (n <= ((size_t)1 << 16)) return modulus != 0;
    return n <= ((size_t)1 << 20) && modulus != 0;
}

static int word_ntt_host(uint64_t* coeffs, size_t n, uint64_t modulus, uint64_t root, bool inverse) {
    if (!word_ntt_args_ok(coeffs, n, modulus)) return KB200_CRYPTO_ERR_INPUT;
    if (n == 1) return KB200_CRYPTO_OK;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_INPUT, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       cudaStream_t st = c->stream;
                       c->d_w.reserve(n * 8, st);
                       c->d_ws.reserve(n * 8, st);
                       KB_CUDA(cudaMemcpyAsync(c->d_w.ptr, coeffs, n * 8, cudaMemcpyHostToDevice, st));
                       const int rc = word_ntt_device(c->wntt_get(), c->d_w.as<uint64_t>(),
                                                      c->d_ws.as<uint64_t>(), n, modulus, root,
                                                      inverse, st);
                       if (rc != 0) return KB200_CRYPTO_ERR_INPUT;
                       KB_CUDA(cudaMemcpyAsync(coeffs, c->d_w.ptr, n * 8, cudaMemcpyDeviceToHost, st));
                       KB_CUDA(cudaStreamSynchronize(st));
                       return KB200_CRYPTO_OK;
                   });
}

// ---- EIP-2537 G1 MSM -------------------------------------------------------

// bls12_381_g1_msm (bls/c-abi/c_bls_pairing.cpp:106-110): 1 = result
// written, 0 = invalid input.  Reference behaviour kept: (0,0) entries are
// infinity and skipped, an input of no finite points gives (0,0).
static int g1_msm_eip2537_host(uint8_t* rx, uint8_t* ry, const uint8_t* xycs, size_t size) {
    if (!rx || !ry || (size && !xycs) || size % 160) return 0;
    const size_t n = size / 160;
    return guarded(KB200_CRYPTO_ERR_BACKEND, 0, KB200_CRYPTO_ERR_INTERNAL, [&]() -> int {
        DeviceCtx* c = get_ctx();
        std::lock_guard<std::mutex> lk(c->mu);
        cudaStream_t st = c->stream;
        c->d_e_in.reserve(size + 16, st);
        c->d_e_tab.reserve(2 * n * (size_t)table_words(2) * 4 + 16, st);  // + GLV rows
        c->d_e_sc.reserve(n * 32 + 16, st);
        c->d_e_out.reserve(256, st);
        c->h_out.reserve(256, st);
        if (size)
            KB_CUDA(cudaMemcpyAsync(c->d_e_in.ptr, xycs, size, cudaMemcpyHostToDevice, st));
        uint8_t* d_out = c->d_e_out.as<uint8_t>();
        uint32_t* d_flag = reinterpret_cast<uint32_t*>(d_out + 128);
        g1_msm_eip2537_device(c->msm_for(2), c->d_e_in.as<uint8_t>(), n, c->d_e_tab.as<uint32_t>(),
                              c->d_e_sc.as<uint8_t>(), d_flag, d_out, st);
        KB_CUDA(cudaMemcpyAsync(c->h_out.ptr, d_out, 132, cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaStreamSynchronize(st));
        const uint8_t* h = static_cast<const uint8_t*>(c->h_out.ptr);
        uint32_t flag;
        std::memcpy(&flag, h + 128, 4);
        if (flag) {
            set_last_error("bls12_381_g1_msm: a point is out of range, off the curve or not in G1");
            return 0;
        }
        std::memset(rx, 0, 16);
        std::memset(ry, 0, 16);
        std::memcpy(rx + 16, h, 48);
        std::memcpy(ry + 16, h + 48, 48);
        return 1;
    });
}

// ---- EIP-4844 blobs ----------------------------------------------------------

// Layout of the blob-op staging buffer d_bl.
constexpr size_t BL_BLOB = 0, BL_Z = BLOB_BYTES, BL_OUT = BLOB_BYTES + 64, BL_Y = BL_OUT + 64,
                 BL_FLAG = BL_Y + 64, BL_SIZE = BL_FLAG + 64;

static void blob_stage(DeviceCtx* c, cudaStream_t st) {
    c->d_bl.reserve(BL_SIZE + (size_t)BLOB_N * 48, st);  // + setup points after BL_SIZE
    c->h_out.reserve(256, st);
}

static int blob_setup_host(const uint8_t* points48, size_t n) {
    if (!points48) return KB200_CRYPTO_ERR_INPUT;
    if (n != BLOB_N) return KB200_CRYPTO_ERR_LENGTH;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       cudaStream_t st = c->stream;
                       blob_stage(c, st);
                       uint8_t* base = c->d_bl.as<uint8_t>();
                       KB_CUDA(cudaMemcpyAsync(base + BL_SIZE, points48, n * 48, cudaMemcpyHostToDevice,
                                               st));
                       uint32_t* d_flag = reinterpret_cast<uint32_t*>(base + BL_FLAG);
                       blob_setup_load_lagrange(c->blob_get(), base + BL_SIZE, d_flag, st);
                       KB_CUDA(cudaMemcpyAsync(c->h_out.ptr, d_flag, 4, cudaMemcpyDeviceToHost, st));
                       KB_CUDA(cudaStreamSynchronize(st));
                       uint32_t flag;
                       std::memcpy(&flag, c->h_out.ptr, 4);
                       if (flag) {
                           blob_setup_mark(c->blob, false);
                           set_last_error("kzg blob setup: a point is not a valid compressed G1 point");
                           return KB200_CRYPTO_ERR_INPUT;
                       }
                       return KB200_CRYPTO_OK;
                   });
}

// kzg_blob_to_commit (kzg/c-abi/c_kzg_blob.cpp:26-30) and kzg_commit_to_proof
// (:32-43).  CRYPTO_ERR_INPUT for null pointers, a blob element or z not
// below r, or no resident setup (the reference's setup-load failure).
static int blob_op_host(const uint8_t* blob, const uint8_t* z, uint8_t* out48, uint8_t* y32) {
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_INPUT, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       if (!blob_setup_ready(c->blob)) {
                           set_last_error("kzg blob ops: no setup loaded (kzg_blob_setup_load_g1_lagrange)");
                           return KB200_CRYPTO_ERR_INPUT;
                       }
                       cudaStream_t st = c->stream;
                       blob_stage(c, st);
                       uint8_t* base = c->d_bl.as<uint8_t>();
                       uint32_t* d_flag = reinterpret_cast<uint32_t*>(base + BL_FLAG);
                       KB_CUDA(cudaMemcpyAsync(base + BL_BLOB, blob, BLOB_BYTES, cudaMemcpyHostToDevice, st));
                       if (z) {
                           KB_CUDA(cudaMemcpyAsync(base + BL_Z, z, 32, cudaMemcpyHostToDevice, st));
                           blob_proof_device(c->blob, c->msm_for(2), base + BL_BLOB, base + BL_Z,
                                             base + BL_OUT, base + BL_Y, d_flag, st);
                       } else {
                           blob_commit_device(c->blob, c->msm_for(2), base + BL_BLOB, base + BL_OUT,
                                              d_flag, st);
                       }
                       // out (48) | pad | y (32) | pad | flag, copied back in one piece
                       KB_CUDA(cudaMemcpyAsync(c->h_out.ptr, base + BL_OUT, BL_FLAG + 4 - BL_OUT,
                                               cudaMemcpyDeviceToHost, st));
                       KB_CUDA(cudaStreamSynchronize(st));
                       const uint8_t* h = static_cast<const uint8_t*>(c->h_out.ptr);
                       uint32_t flag;
                       std::memcpy(&flag, h + (BL_FLAG - BL_OUT), 4);
                       if (flag) {
                           set_last_error("kzg blob ops: a field element is not below r");
                           return KB200_CRYPTO_ERR_INPUT;
                       }
                       std::memcpy(out48, h, 48);
                       if (y32) std::memcpy(y32, h + (BL_Y - BL_OUT), 32);
                       return KB200_CRYPTO_OK;
                   });
}

// ---- KZG -------------------------------------------------------------------

static void commit_on_device(DeviceCtx* c, uint32_t* d_evals, size_t n, uint8_t* d_out48,
                             cudaStream_t st) {
    if (!is_pow2(n)) throw std::invalid_argument("kzg: n must be a power of two");
    if (n > c->srs_n) throw std::invalid_argument("kzg: SRS shorter than the polynomial");
    ntt_run(c->ntt_for(2), d_evals, n, /*inverse=*/1, /*coset=*/0, 1, st);
    c->d_tmp.reserve(256, st);
    MsmOptions opt;
    const uint32_t* table = c->d_srs.as<uint32_t>();
    const int sc = shift_c_for(&n, 1);
    if (const uint32_t* t = shift_tables_get(c->srs_shift_get(), sc, st)) {
        opt.shift_c = sc;
        opt.shift_stride = c->srs_n;
        table = t;
    }
    msm_run_table(c->msm_for(2), reinterpret_cast<const uint8_t*>(d_evals), table, n,
                  c->d_tmp.as<uint8_t>(), d_out48, st, opt);
}

// Autotuner step for single commits against the resident SRS: for each size
// class 2^lg (lg in [log_lo, log_hi], at most the SRS length) time one
// commit per shifted-table window 13 / 16 / 19 and keep the fastest in the
// commit tuning table.  Appends "<key> commit 2 <lg> <c> <ms>" lines to log.
// Returns the classes tuned (0 without a resident SRS).
int tune_commit_windows(int log_lo, int log_hi, const std::string& key, std::string& log) {
    DeviceCtx* c = get_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->srs_n) return 0;
    cudaStream_t st = c->stream;
    int tuned = 0;
    const size_t nmax = std::min(c->srs_n, (size_t)1 << log_hi);
    std::vector<uint8_t> hs(nmax * 32);
    kb200_gen_scalars(2, 0xC0117u, nmax, 0, hs.data());
    DevBuf src;
    src.reserve(nmax * 32, st);
    c->d_a.reserve(nmax * 32 + 64, st);
    c->d_out.reserve(256, st);
    KB_CUDA(cudaMemcpyAsync(src.ptr, hs.data(), nmax * 32, cudaMemcpyHostToDevice, st));
    cudaEvent_t a, b;
    KB_CUDA(cudaEventCreate(&a));
    KB_CUDA(cudaEventCreate(&b));
    for (int lg = log_lo; lg <= log_hi && ((size_t)1 << lg) <= c->srs_n; ++lg) {
        const size_t n = (size_t)1 << lg;
        int best_c = 0;
        float best = 1e30f;
        for (int cand : {13, 16, 19}) {
            commit_tune_set(lg, cand);
            auto one = [&] {
                KB_CUDA(cudaMemcpyAsync(c->d_a.ptr, src.ptr, n * 32, cudaMemcpyDeviceToDevice, st));
                commit_on_device(c, c->d_a.as<uint32_t>(), n, c->d_out.as<uint8_t>(), st);
            };
            one();  // builds the window's shifted table and sizes the engines
            KB_CUDA(cudaStreamSynchronize(st));
            const int reps = lg >= 14 ? 3 : 8;
            KB_CUDA(cudaEventRecord(a, st));
            for (int r = 0; r < reps; ++r) one();
            KB_CUDA(cudaEventRecord(b, st));
            KB_CUDA(cudaEventSynchronize(b));
            float ms = 0;
            KB_CUDA(cudaEventElapsedTime(&ms, a, b));
            ms /= reps;
            if (ms < best) {
                best = ms;
                best_c = cand;
            }
        }
        commit_tune_set(lg, best_c);
        log += key + " commit 2 " + std::to_string(lg) + " " + std::to_string(best_c) + " " +
               std::to_string(best) + "\n";
        ++tuned;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    KB_CUDA(cudaStreamSynchronize(st));
    src.release();
    return tuned;
}

// After a new SRS: build the shifted tables of every window size a commit of
// up to srs_n evaluations selects, and run one commit of zeros per power of
// two, so the per-call engines reach their working size here.  Without it the
// first commit of each size class paid for its table build and for engine
// growth (single allocations took up to ~90 ms on a B200), which set
// per-call throughput anywhere from 280 to 990 commits/s between runs.
static void srs_prepare_commits(DeviceCtx* c, cudaStream_t st) {
    const size_t n = c->srs_n;
    if (n == 0) return;
    std::set<int> cs;
    for (size_t m = 1; m <= n; m <<= 1) cs.insert(shift_c_for(&m, 1));
    for (int sc : cs) shift_tables_get(c->srs_shift_get(), sc, st);
    c->d_a.reserve(n * 32 + 64, st);
    c->d_out.reserve(256, st);
    KB_CUDA(cudaMemsetAsync(c->d_a.ptr, 0, n * 32, st));
    for (size_t m = 1; m <= n; m <<= 1)
        commit_on_device(c, c->d_a.as<uint32_t>(), m, c->d_out.as<uint8_t>(), st);
    KB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace kb200

using namespace kb200;

extern "C" {

int gpukit_multi_pippenger(uint32_t curve, const uint8_t* scalars, const uint8_t* points, size_t n,
                           uint8_t* result) {
    return msm_host(curve, scalars, points, n, result, false);
}

int gpukit_multi_pippenger_cuda(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
                                size_t n, uint8_t* result) {
    return msm_host(curve, scalars, points, n, result, false);
}

int gpukit_multi_pippenger_subgroup(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
                                    size_t n, uint8_t* result) {
    return msm_host(curve, scalars, points, n, result, true);
}

int ntt_fr_forward(int curve, uint8_t* coeffs32le, size_t n, int coset) {
    return ntt_host(curve, coeffs32le, n, 0, coset);
}

int ntt_fr_inverse(int curve, uint8_t* coeffs32le, size_t n, int coset) {
    return ntt_host(curve, coeffs32le, n, 1, coset);
}

int kzg_srs_load_g1(const uint8_t* points96be, size_t n) {
    if (!points96be && n) return KB200_CRYPTO_ERR_INPUT;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       cudaStream_t st = c->stream;
                       c->d_b.reserve(n * 96 + 16, st);
                       c->d_srs.reserve(n * (size_t)table_words(2) * 4 + 16, st);
                       if (n) {
                           KB_CUDA(cudaMemcpyAsync(c->d_b.ptr, points96be, n * 96,
                                                   cudaMemcpyHostToDevice, st));
                           points_wire_to_table(2, c->d_b.as<uint8_t>(), c->d_srs.as<uint32_t>(), n, st);
                       }
                       KB_CUDA(cudaStreamSynchronize(st));
                       c->srs_n = n;
                       shift_tables_reset(c->srs_shift_get(), c->d_srs.as<uint32_t>(), n);
                       srs_prepare_commits(c, st);
                       return KB200_CRYPTO_OK;
                   });
}

int kzg_srs_generate_g1(const uint8_t tau32le[32], size_t n) {
    if (!tau32le) return KB200_CRYPTO_ERR_INPUT;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       cudaStream_t st = c->stream;
                       c->d_a.reserve(n * 32 + 64, st);
                       c->d_srs.reserve(n * (size_t)table_words(2) * 4 + 16, st);
                       uint8_t* d_tau = c->d_a.as<uint8_t>() + n * 32;
                       KB_CUDA(cudaMemcpyAsync(d_tau, tau32le, 32, cudaMemcpyHostToDevice, st));
                       fr_powers(2, d_tau, n, c->d_a.as<uint8_t>(), st);
                       fixed_base_mul(c->fb_for(2), c->d_a.as<uint8_t>(), n, c->d_srs.as<uint32_t>(),
                                      nullptr, st);
                       KB_CUDA(cudaStreamSynchronize(st));
                       c->srs_n = n;
                       shift_tables_reset(c->srs_shift_get(), c->d_srs.as<uint32_t>(), n);
                       srs_prepare_commits(c, st);
                       return KB200_CRYPTO_OK;
                   });
}

int kzg_srs_read_g1(uint8_t* points96be, size_t offset, size_t count) {
    if (!points96be && count) return KB200_CRYPTO_ERR_INPUT;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       if (offset + count > c->srs_n) return KB200_CRYPTO_ERR_LENGTH;
                       cudaStream_t st = c->stream;
                       c->d_b.reserve(count * 96 + 16, st);
                       points_table_to_wire(2, c->d_srs.as<uint32_t>() + offset * table_words(2),
                                            c->d_b.as<uint8_t>(), count, st);
                       KB_CUDA(cudaMemcpyAsync(points96be, c->d_b.ptr, count * 96,
                                               cudaMemcpyDeviceToHost, st));
                       KB_CUDA(cudaStreamSynchronize(st));
                       return KB200_CRYPTO_OK;
                   });
}

size_t kzg_srs_size(void) {
    try {
        DeviceCtx* c = get_ctx();
        std::lock_guard<std::mutex> lk(c->mu);
        return c->srs_n;
    } catch (...) {
        return 0;
    }
}

int kzg_commit_fr(const uint8_t* evals32le, size_t n, uint8_t commit48[48]) {
    if (!evals32le || !commit48) return KB200_CRYPTO_ERR_INPUT;
    if (!is_pow2(n)) return KB200_CRYPTO_ERR_LENGTH;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       if (n > c->srs_n) return KB200_CRYPTO_ERR_LENGTH;
                       cudaStream_t st = c->stream;
                       c->d_a.reserve(n * 32 + 16, st);
                       c->d_out.reserve(256, st);
                       c->h_out.reserve(256, st);
                       KB_CUDA(cudaMemcpyAsync(c->d_a.ptr, evals32le, n * 32,
                                               cudaMemcpyHostToDevice, st));
                       commit_on_device(c, c->d_a.as<uint32_t>(), n, c->d_out.as<uint8_t>(), st);
                       KB_CUDA(cudaMemcpyAsync(c->h_out.ptr, c->d_out.ptr, 48,
                                               cudaMemcpyDeviceToHost, st));
                       KB_CUDA(cudaStreamSynchronize(st));
                       std::memcpy(commit48, c->h_out.ptr, 48);
                       return KB200_CRYPTO_OK;
                   });
}

int kzg_commit_batch(const uint8_t* evals32le, const size_t* sizes, size_t count,
                     uint8_t* commits48) {
    if (count && (!evals32le || !sizes || !commits48)) return KB200_CRYPTO_ERR_INPUT;
    for (size_t i = 0; i < count; ++i)
        if (!is_pow2(sizes[i])) return KB200_CRYPTO_ERR_LENGTH;
    if (count == 0) return KB200_CRYPTO_OK;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       for (size_t i = 0; i < count; ++i)
                           if (sizes[i] > c->srs_n) return KB200_CRYPTO_ERR_LENGTH;
                       commit_batch_host(c->batcher_get(), evals32le, sizes, count,
                                         c->d_srs.as<uint32_t>(), c->srs_n, commits48, c->stream,
                                         /*use_graph=*/true);
                       return KB200_CRYPTO_OK;
                   });
}

static int msm_device(uint32_t curve, const void* d_scalars, const void* d_points, size_t n,
                      void* d_result, void* stream, bool points_in_g1) {
    if (!d_result || (n && (!d_scalars || !d_points))) return KB200_GPUKIT_ERR_NULL_ARG;
    if (curve != 1 && curve != 2) return KB200_GPUKIT_ERR_BACKEND;
    return guarded(KB200_GPUKIT_ERR_DISPATCH, KB200_GPUKIT_ERR_BAD_SIZE, KB200_GPUKIT_ERR_DISPATCH,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       MsmOptions opt;
                       opt.ref_carry_quirk = true;
                       opt.points_in_g1 = points_in_g1;
                       msm_run_wire(c->msm_for((int)curve), (const uint8_t*)d_scalars,
                                    (const uint8_t*)d_points, n, (uint8_t*)d_result, nullptr,
                                    (cudaStream_t)stream, opt);
                       return KB200_GPUKIT_OK;
                   });
}

int kb200_msm_device(uint32_t curve, const void* d_scalars, const void* d_points, size_t n,
                     void* d_result, void* stream) {
    return msm_device(curve, d_scalars, d_points, n, d_result, stream, false);
}

int kb200_msm_device_subgroup(uint32_t curve, const void* d_scalars, const void* d_points,
                              size_t n, void* d_result, void* stream) {
    return msm_device(curve, d_scalars, d_points, n, d_result, stream, true);
}

int kzg_blob_setup_load_g1_lagrange(const uint8_t* points48, size_t n) {
    return blob_setup_host(points48, n);
}

int kzg_blob_setup_generate(const uint8_t tau32le[32]) {
    if (!tau32le) return KB200_CRYPTO_ERR_INPUT;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       cudaStream_t st = c->stream;
                       blob_stage(c, st);
                       uint8_t* d_tau = c->d_bl.as<uint8_t>() + BL_Z;
                       KB_CUDA(cudaMemcpyAsync(d_tau, tau32le, 32, cudaMemcpyHostToDevice, st));
                       blob_setup_generate(c->blob_get(), c->fb_for(2), d_tau, st);
                       KB_CUDA(cudaStreamSynchronize(st));
                       return KB200_CRYPTO_OK;
                   });
}

int kzg_blob_to_commit(const uint8_t blob[131072], uint8_t commit[48]) {
    if (!blob || !commit) return KB200_CRYPTO_ERR_INPUT;
    return blob_op_host(blob, nullptr, commit, nullptr);
}

int kzg_commit_to_proof(const uint8_t blob[131072], const uint8_t z[32], uint8_t proof[48],
                        uint8_t y[32]) {
    if (!blob || !z || !proof || !y) return KB200_CRYPTO_ERR_INPUT;
    return blob_op_host(blob, z, proof, y);
}

int bls12_381_g1_msm(uint8_t rx[64], uint8_t ry[64], const uint8_t* xycs, size_t size) {
    return g1_msm_eip2537_host(rx, ry, xycs, size);
}

int kb200_bls12_381_g1_msm_device(const void* d_xycs, size_t size, void* d_out_wire96,
                                  void* d_status, void* stream) {
    if (!d_out_wire96 || !d_status || (size && !d_xycs) || size % 160) return KB200_CRYPTO_ERR_INPUT;
    const size_t n = size / 160;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       cudaStream_t st = (cudaStream_t)stream;
                       c->d_e_tab.reserve(2 * n * (size_t)table_words(2) * 4 + 16, st);  // + GLV rows
                       c->d_e_sc.reserve(n * 32 + 16, st);
                       g1_msm_eip2537_device(c->msm_for(2), (const uint8_t*)d_xycs, n,
                                             c->d_e_tab.as<uint32_t>(), c->d_e_sc.as<uint8_t>(),
                                             (uint32_t*)d_status, (uint8_t*)d_out_wire96, st);
                       return KB200_CRYPTO_OK;
                   });
}

int ntt_forward(uint64_t* coeffs, size_t n, uint64_t modulus, uint64_t root) {
    return word_ntt_host(coeffs, n, modulus, root, false);
}

int ntt_inverse(uint64_t* coeffs, size_t n, uint64_t modulus, uint64_t root_inv) {
    return word_ntt_host(coeffs, n, modulus, root_inv, true);
}

int kb200_word_ntt_device(void* d_coeffs, void* d_scratch, size_t n, uint64_t modulus,
                          uint64_t root, int inverse, void* stream) {
    if (!word_ntt_args_ok((const uint64_t*)d_coeffs, n, modulus)) return KB200_CRYPTO_ERR_INPUT;
    if (n > ((size_t)1 << 11) && n <= ((size_t)1 << 16) && !d_scratch) return KB200_CRYPTO_ERR_INPUT;
    if (n == 1) return KB200_CRYPTO_OK;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_INPUT, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       const int rc = word_ntt_device(c->wntt_get(), (uint64_t*)d_coeffs,
                                                      (uint64_t*)d_scratch, n, modulus, root,
                                                      inverse != 0, (cudaStream_t)stream);
                       return rc == 0 ? KB200_CRYPTO_OK : KB200_CRYPTO_ERR_INPUT;
                   });
}

int kb200_ntt_device(int curve, void* d_data, size_t n, int inverse, int coset, size_t batch,
                     void* stream) {
    if (!d_data) return KB200_CRYPTO_ERR_INPUT;
    if (curve != 1 && curve != 2) return KB200_CRYPTO_ERR_INPUT;
    if (!is_pow2(n) || n > ((size_t)1 << ntt_max_log(curve))) return KB200_CRYPTO_ERR_LENGTH;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       ntt_run(c->ntt_for(curve), (uint32_t*)d_data, n, inverse, coset, batch,
                               (cudaStream_t)stream);
                       return KB200_CRYPTO_OK;
                   });
}

int kb200_g1_fixed_base_device(uint32_t curve, const void* d_scalars, size_t n,
                               void* d_out_points, void* stream) {
    if (n && (!d_scalars || !d_out_points)) return KB200_GPUKIT_ERR_NULL_ARG;
    if (curve != 1 && curve != 2) return KB200_GPUKIT_ERR_BACKEND;
    return guarded(KB200_GPUKIT_ERR_DISPATCH, KB200_GPUKIT_ERR_BAD_SIZE, KB200_GPUKIT_ERR_DISPATCH,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       FixedBase* fb = c->fb_for((int)curve);
                       fixed_base_mul(fb, (const uint8_t*)d_scalars, n, nullptr,
                                      (uint8_t*)d_out_points, (cudaStream_t)stream);
                       return KB200_GPUKIT_OK;
                   });
}

int kb200_fr_powers_device(int curve, const void* d_tau, size_t n, void* d_out, void* stream) {
    if (n && (!d_tau || !d_out)) return KB200_CRYPTO_ERR_INPUT;
    if (curve != 1 && curve != 2) return KB200_CRYPTO_ERR_INPUT;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       fr_powers(curve, (const uint8_t*)d_tau, n, (uint8_t*)d_out,
                                 (cudaStream_t)stream);
                       return KB200_CRYPTO_OK;
                   });
}

int kb200_kzg_commit_device(void* d_evals, size_t n, void* d_commit48, void* stream) {
    if (!d_evals || !d_commit48) return KB200_CRYPTO_ERR_INPUT;
    return guarded(KB200_CRYPTO_ERR_BACKEND, KB200_CRYPTO_ERR_LENGTH, KB200_CRYPTO_ERR_INTERNAL,
                   [&]() -> int {
                       DeviceCtx* c = get_ctx();
                       std::lock_guard<std::mutex> lk(c->mu);
                       commit_on_device(c, (uint32_t*)d_evals, n, (uint8_t*)d_commit48,
                                        (cudaStream_t)stream);
                       return KB200_CRYPTO_OK;
                   });
}

const char* kb200_last_error(void) { return g_last_error.c_str(); }

int kb200_device_available(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count > 0 ? 1 : 0;
}

unsigned long long kb200_launch_count(void) { return g_launches.load(); }

void kb200_profile_enable(int on) { g_profile.store(on != 0); }

int kb200_msm_stage_ms(uint32_t curve, float* out, int max) {
    if (!out || max <= 0 || (curve != 1 && curve != 2)) return -1;
    try {
        DeviceCtx* c = get_ctx();
        std::lock_guard<std::mutex> lk(c->mu);
        if (!c->msm[curve]) return 0;
        return msm_stage_ms(c->msm[curve], out, max);
    } catch (...) {
        return -1;
    }
}

static double msm_entries(uint32_t curve, size_t n, bool in_g1) {
    MsmOptions opt;
    opt.points_in_g1 = in_g1;
    if (curve != 1 && curve != 2) return 0.0;
    if (msm_wire_uses_glv((int)curve, opt)) {
        const MsmPlan p = make_msm_plan_glv((int)curve, n, opt);
        // populated windows of the halves: their magnitudes are below 2^128 / 2^126
        const int hb = curve == 2 ? 128 : 126;
        return 2.0 * (double)n * (double)((hb + p.c - 1) / p.c) * (1.0 - std::ldexp(1.0, -p.c));
    }
    const MsmPlan p = make_msm_plan((int)curve, n, opt);
    return (double)n * (double)((255 + p.c - 1) / p.c) * (1.0 - std::ldexp(1.0, -p.c));
}

static int msm_window(uint32_t curve, size_t n, bool in_g1) {
    MsmOptions opt;
    opt.points_in_g1 = in_g1;
    if (curve != 1 && curve != 2) return 0;
    if (msm_wire_uses_glv((int)curve, opt)) return make_msm_plan_glv((int)curve, n, opt).c;
    return make_msm_plan((int)curve, n, opt).c;
}

double kb200_msm_entries(uint32_t curve, size_t n) { return msm_entries(curve, n, false); }
double kb200_msm_entries_subgroup(uint32_t curve, size_t n) { return msm_entries(curve, n, true); }
int kb200_msm_window(uint32_t curve, size_t n) { return msm_window(curve, n, false); }
int kb200_msm_window_subgroup(uint32_t curve, size_t n) { return msm_window(curve, n, true); }

}  // extern "C"
