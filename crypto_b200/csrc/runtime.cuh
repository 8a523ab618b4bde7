// Host-side runtime pieces shared by the kernels: error handling, grow-only
// scratch buffers, and a device prefix sum.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace kb200 {

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* what) : std::runtime_error(what), code(c) {}
};

#define KB_CUDA(expr)                                                              \
    do {                                                                           \
        cudaError_t kb_err_ = (expr);                                              \
        if (kb_err_ != cudaSuccess) {                                              \
            char kb_buf_[256];                                                     \
            std::snprintf(kb_buf_, sizeof kb_buf_, "%s failed: %s (%s:%d)", #expr, \
                          cudaGetErrorString(kb_err_), __FILE__, __LINE__);        \
            throw ::kb200::CudaError(kb_err_, kb_buf_);                            \
        }                                                                          \
    } while (0)

// Every kernel launch site calls KB_LAUNCH_CHECK(): it checks the launch and
// counts it (kb200_launch_count() reports the total, so a benchmark can state
// how many of this library's kernels ran in its timed region).
void count_launch();
#define KB_LAUNCH_CHECK()             \
    do {                              \
        KB_CUDA(cudaGetLastError());  \
        ::kb200::count_launch();      \
    } while (0)

// Optional per-stage timing (CUDA events on the work stream), off by default.
bool profiling_enabled();

// Records the most recent failure message so the C ABI can report it.
void set_last_error(const std::string& msg);

// KB200_ALLOC_TRACE=1: every device-buffer growth logged on stderr with its
// size and host time.
bool alloc_trace_enabled();
void alloc_trace(size_t from, size_t to, double ms);

// Deferred frees for a thread that owns every stream its buffers are used
// on (the commit server's worker): a buffer that grows on such a thread keeps
// its old allocation in a per-thread list instead of freeing it, because
// cudaFree waits for the whole device (another slot's batch included) and,
// measured under load, sometimes for hundreds of milliseconds more.  The
// thread frees the list with devbuf_free_retired() once its streams are idle
// and the list holds more than a set number of bytes, and when it exits.
inline thread_local bool t_devbuf_defer = false;
inline thread_local std::vector<void*> t_devbuf_retired;
inline thread_local size_t t_devbuf_retired_bytes = 0;
inline void devbuf_defer_frees(bool on) { t_devbuf_defer = on; }
inline size_t devbuf_retired_bytes() { return t_devbuf_retired_bytes; }
inline void devbuf_free_retired() {
    const auto t0 = std::chrono::steady_clock::now();
    for (void* p : t_devbuf_retired) cudaFree(p);
    if (alloc_trace_enabled() && !t_devbuf_retired.empty())
        std::fprintf(stderr, "[devbuf] freed %zu retired buffers (%zu bytes), %.3f ms\n",
                     t_devbuf_retired.size(), t_devbuf_retired_bytes,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    t_devbuf_retired.clear();
    t_devbuf_retired_bytes = 0;
}

// Process-wide count of device allocations replaced or released by DevBuf.
// Work captured into a CUDA graph holds raw device addresses; a graph
// captured when this count had another value may name freed memory and must
// be captured again.
inline std::atomic<unsigned long long> g_devbuf_moves{0};
inline unsigned long long devbuf_moves() { return g_devbuf_moves.load(std::memory_order_acquire); }

// A grow-only device buffer.  Growing synchronises the owning stream first,
// because the old allocation may still be read by queued work (or, on a
// thread with deferred frees, keeps the old allocation until that thread's
// streams are idle).
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    void reserve(size_t need, cudaStream_t stream) {
        if (need <= bytes) return;
        const bool tr = alloc_trace_enabled();
        const auto t0 = std::chrono::steady_clock::now();
        const size_t from = bytes;
        if (ptr) {
            if (t_devbuf_defer) {
                t_devbuf_retired.push_back(ptr);
                t_devbuf_retired_bytes += bytes;
            } else {
                KB_CUDA(cudaStreamSynchronize(stream));
                KB_CUDA(cudaFree(ptr));
            }
            g_devbuf_moves.fetch_add(1, std::memory_order_acq_rel);
            ptr = nullptr;
            bytes = 0;
        }
        // 1/8 headroom; on a deferring thread (a server under load, where an
        // allocation can stall it) half again, so a buffer grows fewer times
        size_t want = need + (t_devbuf_defer ? need / 2 : need / 8) + 256;
        KB_CUDA(cudaMalloc(&ptr, want));
        bytes = want;
        if (tr)
            alloc_trace(from, want,
                        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
    void release() {
        if (ptr) {
            cudaFree(ptr);
            g_devbuf_moves.fetch_add(1, std::memory_order_acq_rel);
        }
        ptr = nullptr;
        bytes = 0;
    }
};

// Pinned host staging buffer (grow-only).
struct HostBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    void reserve(size_t need, cudaStream_t stream) {
        if (need <= bytes) return;
        if (ptr) {
            KB_CUDA(cudaStreamSynchronize(stream));
            KB_CUDA(cudaFreeHost(ptr));
            ptr = nullptr;
            bytes = 0;
        }
        size_t want = need + need / 8 + 256;
        KB_CUDA(cudaMallocHost(&ptr, want));
        bytes = want;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Exclusive prefix sum of n 32-bit values: out[i] = sum_{j<i} f(in[j]) and
// out[n] = total, where f is the identity (div == 0) or ceil(x / div).
// tmp must hold scan_tmp_words(n) words.
size_t scan_tmp_words(size_t n);
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t div,
                        uint32_t* tmp, cudaStream_t stream);
// The same starting from the device value *init (0 if null), the total also
// written to *total_copy (if not null): consecutive ranges of one array
// scanned in turn, each from the previous range's total, without the host.
void exclusive_scan_u32_chained(const uint32_t* in, uint32_t* out, size_t n, uint32_t div,
                                const uint32_t* init, uint32_t* total_copy, uint32_t* tmp,
                                cudaStream_t stream);

inline unsigned ceil_div_u(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace kb200
