// Device exclusive prefix sum over 32-bit counts (bucket offsets, segment
// offsets).  Three phases: per-block scan of 2048-element tiles with warp
// shuffles, a single-block scan of the tile totals, and a fix-up pass.
#include "runtime.cuh"

namespace kb200 {

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 2;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t xform(uint32_t v, uint32_t div) {
    return div ? (v + div - 1) / div : v;
}

// Inclusive block scan of one value per thread; returns the inclusive value,
// writes the block total to *total.
__device__ uint32_t block_inclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += t;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        uint32_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += t;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    if (warp > 0) v += warp_sums[warp - 1];
    if (total) *total = warp_sums[((blockDim.x + 31) >> 5) - 1];
    __syncthreads();
    return v;
}

__global__ void k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                             size_t n, uint32_t div, uint32_t* __restrict__ tile_sums) {
    const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < n) ? xform(in[base + k], div) : 0;
        local += v[k];
    }
    uint32_t total;
    uint32_t incl = block_inclusive_scan(local, &total);
    uint32_t run = incl - local;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Single block: exclusive scan of the tile totals in place, starting from
// *init (0 if null); writes the grand total to out[n] (and to *total_copy).
__global__ void k_scan_sums(uint32_t* __restrict__ sums, unsigned nt, uint32_t* __restrict__ out,
                            size_t n, const uint32_t* __restrict__ init,
                            uint32_t* __restrict__ total_copy) {
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = init ? *init : 0u;
    __syncthreads();
    for (unsigned base = 0; base < nt; base += blockDim.x) {
        unsigned i = base + threadIdx.x;
        uint32_t v = i < nt ? sums[i] : 0;
        uint32_t total;
        uint32_t incl = block_inclusive_scan(v, &total);
        if (i < nt) sums[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[n] = carry;
        if (total_copy) *total_copy = carry;
    }
}

__global__ void k_scan_fix(uint32_t* __restrict__ out, size_t n, const uint32_t* __restrict__ sums) {
    const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    const uint32_t add = sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < n) out[base + k] += add;
}

}  // namespace

size_t scan_tmp_words(size_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t div,
                        uint32_t* tmp, cudaStream_t stream) {
    exclusive_scan_u32_chained(in, out, n, div, nullptr, nullptr, tmp, stream);
}

void exclusive_scan_u32_chained(const uint32_t* in, uint32_t* out, size_t n, uint32_t div,
                                const uint32_t* init, uint32_t* total_copy, uint32_t* tmp,
                                cudaStream_t stream) {
    const unsigned nt = (unsigned)((n + SCAN_TILE - 1) / SCAN_TILE);
    if (nt == 0) {
        if (init || total_copy) {
            k_scan_sums<<<1, SCAN_THREADS, 0, stream>>>(tmp, 0, out, 0, init, total_copy);
            KB_LAUNCH_CHECK();
        } else {
            KB_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t), stream));
        }
        return;
    }
    k_scan_tiles<<<nt, SCAN_THREADS, 0, stream>>>(in, out, n, div, tmp);
    KB_LAUNCH_CHECK();
    k_scan_sums<<<1, SCAN_THREADS, 0, stream>>>(tmp, nt, out, n, init, total_copy);
    KB_LAUNCH_CHECK();
    k_scan_fix<<<nt, SCAN_THREADS, 0, stream>>>(out, n, tmp);
    KB_LAUNCH_CHECK();
}

}  // namespace kb200
