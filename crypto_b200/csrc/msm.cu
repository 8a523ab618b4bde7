// MSM host driver: window plans, batch descriptors, scratch management and
// the launch sequence.  Curve-specific kernels live in msm_kernels.cuh.
#include "msm.cuh"
#include "msm_desc.cuh"
#include "runtime.cuh"

#include <algorithm>
#include <cstdlib>
#include <limits>
#include <map>
#include <mutex>
#include <tuple>

namespace kb200 {

const MsmLaunchers& msm_launchers_bls();
const MsmLaunchers& msm_launchers_bn();
const MsmLaunchers& msm_launchers(int curve) {
    return curve == 2 ? msm_launchers_bls() : msm_launchers_bn();
}

void set_smem_attr(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& have = done[{kernel, dev}];
    if (have >= bytes) return;
    KB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    have = bytes;
}

// ---------------------------------------------------------------------------
// Curve-independent sort kernels
// ---------------------------------------------------------------------------

// Threads of a pairing level with at most `slots` output slots.
static uint32_t pair_threads(unsigned long long slots) {
    return (uint32_t)((slots + PAIR_J - 1) / PAIR_J);
}

// Per-chunk first pairing level: sub-run (c, b) of the chunk-major sort has
// cnt[c B + b] output slots; cntT is the same counts bucket-major.
__global__ void k_transpose_counts(const uint32_t* __restrict__ cnt, uint32_t B, uint32_t CH,
                                   uint32_t* __restrict__ cntT) {
    const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= (size_t)B * CH) return;
    const uint32_t c = (uint32_t)(r / B), b = (uint32_t)(r % B);
    cntT[(size_t)b * CH + c] = cnt[r];
}

// From the bucket-major exclusive scan of the sub-run counts: each sub-run's
// first output row (dst_off, chunk-major index) and each bucket's first row
// (in1, B + 1 entries: the runs the next level reads).
__global__ void k_chunk_offsets(const uint32_t* __restrict__ scanT, uint32_t B, uint32_t CH,
                                uint32_t* __restrict__ dst_off, uint32_t* __restrict__ in1) {
    const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < (size_t)B * CH) {
        const uint32_t c = (uint32_t)(r / B), b = (uint32_t)(r % B);
        dst_off[r] = scanT[(size_t)b * CH + c];
    }
    if (r <= B) in1[r] = scanT[(size_t)r * CH];
}

// cnt[b] = ceil(m_b / 2) for the runs of a pairing level.
__global__ void k_pair_counts(const uint32_t* __restrict__ in_off, uint32_t B, uint32_t* __restrict__ cnt) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < B) cnt[b] = (in_off[b + 1] - in_off[b] + 1) >> 1;
}

// Counting sort of the (key, val) entries in two passes.  Pass 1 counts the
// keys and gives every entry its rank among the entries of its key: a warp's
// lanes with equal keys (match_any) take one atomicAdd for all of them, and
// each lane's rank is that base plus the number of its peers below it.
// Pass 2, after the scan of the counts, writes val to offsets[key] + rank:
// no atomics.  The order inside a bucket is whatever order the atomics
// granted; bucket sums do not depend on it.
// Rank of entry slot t among the entries with its key: the next free place
// of the key's run, by one atomic on its count.  Repeated keys (skewed
// scalars, where one bucket can take millions of entries) show up between
// neighbouring lanes; only then group the warp by key.  Without that, one
// atomic per lane: every atomicAdd returns a distinct rank, so both paths
// are exact.  All lanes of the warp that hold a slot call it together.
__device__ __forceinline__ void rank_entry(const uint32_t* __restrict__ keys, unsigned long long t,
                                           uint32_t* __restrict__ counts,
                                           uint32_t* __restrict__ ranks) {
    const uint32_t key = keys[t];
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const uint32_t up = __shfl_down_sync(mask, key, 1);
    const bool dup = (lane < 31) && ((mask >> (lane + 1)) & 1u) && up == key && key != KEY_SENTINEL;
    if (!__any_sync(mask, dup)) {
        ranks[t] = key != KEY_SENTINEL ? atomicAdd(&counts[key], 1u) : 0u;
        return;
    }
    const unsigned peers = __match_any_sync(mask, key);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader && key != KEY_SENTINEL) base = atomicAdd(&counts[key], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    ranks[t] = base + __popc(peers & ((1u << lane) - 1u));
}

__global__ void k_rank(const uint32_t* __restrict__ keys, unsigned long long total,
                       uint32_t* __restrict__ counts, uint32_t* __restrict__ ranks) {
    const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    rank_entry(keys, t, counts, ranks);
}

// The same over the entries of scalar rows [lo, lo + len) of one MSM of n
// scalars, whose entry slots are g * n + j (entry group g < G: a window, or
// a window of one GLV half; row j): ranking as each chunk of scalars lands.
__global__ void k_rank_rows(const uint32_t* __restrict__ keys, uint32_t n, uint32_t G, uint32_t lo,
                            uint32_t len, uint32_t* __restrict__ counts,
                            uint32_t* __restrict__ ranks) {
    const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned long long)G * len) return;
    const uint32_t g = (uint32_t)(t / len), j = lo + (uint32_t)(t % len);
    rank_entry(keys, (unsigned long long)g * n + j, counts, ranks);
}

// ---- Tiled ranking (one MSM whose windows have at most RANK_TILE_M buckets) --
// A tile is a row range of one entry group (window, or window of a GLV half)
// within one row chunk: all its keys lie in one window's bucket range, so its
// block counts them in shared memory (local ranks), reserves each bucket's
// places with one global atomic per distinct bucket (at n = 2^22 with 16-bit
// windows, a tile of ~440 K entries over 32 K buckets: ~14x fewer global
// atomics than one per entry), then adds the reserved base to every local
// rank, so the plain scatter (offsets[key] + rank) follows.  Entries whose
// key falls outside the tile's counter range (the GLV top window's buckets
// past M) take a global atomic each.  Each thread handles RANK_TILE_U
// entries per round, their loads issued together.
constexpr uint32_t RANK_TILE_M = 32768;          // shared-memory counters per tile (128 KiB)
constexpr uint32_t RANK_GLOBAL = 0x80000000u;    // rank taken from the global count
constexpr int RANK_TILE_THREADS = 1024;
constexpr int RANK_TILE_U = 4;

struct RankTiles {
    uint32_t n;             // scalars (rows); entry slot g * n + j
    uint32_t G;             // entry groups
    uint32_t TS;            // rows per row chunk
    uint32_t R;             // rows per tile
    uint32_t Q;             // tiles per (chunk, group)
    uint32_t M;             // counters per tile (the window's bucket count)
    uint32_t glv;           // groups 2w + h share window w
    uint32_t bucket_base;   // the item's first bucket
    uint32_t chunk_rows;    // chunk-major keys: rows per key chunk (0: none)
    uint32_t chunk_stride;  // keys per key chunk
};

// Grid (G Q) per row chunk, chunks c0, c0 + 1, ... (blockIdx.y).
__global__ void __launch_bounds__(RANK_TILE_THREADS) k_rank_tiles(const uint32_t* __restrict__ keys,
                                                                  RankTiles t, uint32_t c0,
                                                                  uint32_t* __restrict__ counts,
                                                                  uint32_t* __restrict__ ranks) {
    extern __shared__ uint32_t sc[];
    const uint32_t c = c0 + blockIdx.y;
    const uint32_t g = blockIdx.x / t.Q, q = blockIdx.x % t.Q;
    const uint32_t kb = (t.chunk_rows ? c * t.chunk_stride : 0u) + t.bucket_base + (t.glv ? g >> 1 : g) * t.M;
    const uint32_t chunk_end = min(t.n, (c + 1) * t.TS);
    const uint32_t r0 = min(chunk_end, c * t.TS + q * t.R), r1 = min(chunk_end, r0 + t.R);
    const unsigned long long gbase = (unsigned long long)g * t.n;
    for (uint32_t k = threadIdx.x; k < t.M; k += blockDim.x) sc[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    constexpr uint32_t STEP = RANK_TILE_THREADS * RANK_TILE_U;
    // local ranks (or global ones, flagged); every lane of a warp runs every
    // round (lanes past the tile's end carry the sentinel key)
    for (uint32_t j0 = r0; j0 < r1; j0 += STEP) {
        uint32_t key[RANK_TILE_U];
#pragma unroll
        for (int u = 0; u < RANK_TILE_U; ++u) {
            const uint32_t j = j0 + u * RANK_TILE_THREADS + threadIdx.x;
            key[u] = j < r1 ? keys[gbase + j] : KEY_SENTINEL;
        }
#pragma unroll
        for (int u = 0; u < RANK_TILE_U; ++u) {
            const uint32_t j = j0 + u * RANK_TILE_THREADS + threadIdx.x;
            const uint32_t kl = key[u] - kb;
            const bool local = kl < t.M;
            const uint32_t up = __shfl_down_sync(0xffffffffu, key[u], 1);
            const bool dup = lane < 31 && up == key[u] && key[u] != KEY_SENTINEL;
            uint32_t r = 0;
            if (!__any_sync(0xffffffffu, dup)) {
                if (key[u] != KEY_SENTINEL)
                    r = local ? atomicAdd(&sc[kl], 1u) : (atomicAdd(&counts[key[u]], 1u) | RANK_GLOBAL);
            } else {
                // repeated keys between neighbouring lanes (skewed scalars):
                // one atomic per group of equal keys
                const unsigned peers = __match_any_sync(0xffffffffu, key[u]);
                const int leader = __ffs(peers) - 1;
                uint32_t b = 0;
                if (lane == leader && key[u] != KEY_SENTINEL) {
                    const uint32_t cnt = (uint32_t)__popc(peers);
                    b = local ? atomicAdd(&sc[kl], cnt) : atomicAdd(&counts[key[u]], cnt);
                }
                b = __shfl_sync(0xffffffffu, b, leader);
                r = b + __popc(peers & ((1u << lane) - 1u));
                if (!local) r |= RANK_GLOBAL;
            }
            if (j < r1) ranks[gbase + j] = r;
        }
    }
    __syncthreads();
    // one reservation per bucket the tile uses; the counter becomes its base
    for (uint32_t k = threadIdx.x; k < t.M; k += blockDim.x) {
        const uint32_t cnt = sc[k];
        sc[k] = cnt ? atomicAdd(&counts[kb + k], cnt) : 0u;
    }
    __syncthreads();
    // rank within the bucket's run
    for (uint32_t j0 = r0; j0 < r1; j0 += STEP) {
        uint32_t key[RANK_TILE_U], r[RANK_TILE_U];
#pragma unroll
        for (int u = 0; u < RANK_TILE_U; ++u) {
            const uint32_t j = j0 + u * RANK_TILE_THREADS + threadIdx.x;
            key[u] = j < r1 ? keys[gbase + j] : KEY_SENTINEL;
            r[u] = j < r1 ? ranks[gbase + j] : 0u;
        }
#pragma unroll
        for (int u = 0; u < RANK_TILE_U; ++u) {
            const uint32_t j = j0 + u * RANK_TILE_THREADS + threadIdx.x;
            if (j >= r1 || key[u] == KEY_SENTINEL) continue;
            ranks[gbase + j] = (r[u] & RANK_GLOBAL) ? (r[u] & ~RANK_GLOBAL) : sc[key[u] - kb] + r[u];
        }
    }
}

__global__ void k_scatter(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                          const uint32_t* __restrict__ ranks, unsigned long long total,
                          const uint32_t* __restrict__ offsets, uint32_t* __restrict__ sorted) {
    const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const uint32_t key = keys[t];
    if (key == KEY_SENTINEL) return;
    sorted[offsets[key] + ranks[t]] = vals[t];
}

// k_scatter over the entries of scalar rows [lo, lo + len) of one MSM of n
// scalars (slots g * n + j, as k_rank_rows).
// offsets is indexed by key + shift (the pipeline's chunk c keeps its B + 1
// offsets at c (B + 1), its keys being c B .. c B + B - 1: shift = c).
__global__ void k_scatter_rows(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                               const uint32_t* __restrict__ ranks, uint32_t n, uint32_t G, uint32_t lo,
                               uint32_t len, const uint32_t* __restrict__ offsets, uint32_t shift,
                               uint32_t* __restrict__ sorted) {
    const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned long long)G * len) return;
    const uint32_t g = (uint32_t)(t / len), j = lo + (uint32_t)(t % len);
    const unsigned long long slot = (unsigned long long)g * n + j;
    const uint32_t key = keys[slot];
    if (key == KEY_SENTINEL) return;
    sorted[offsets[key + shift] + ranks[slot]] = vals[slot];
}

// Host-input pipeline, level 1 after the per-chunk first level: chunk c's
// offsets are off[c (B + 1) + b], b <= B, and its first-level sums of
// bucket b sit at rows off[c (B + 1) + b] .. + ceil(len / 2) (the sub-run's
// own entry positions).  tot[b] = the bucket's sums over the
// chunks; idx lists them bucket by bucket (chunk by chunk inside a bucket),
// so level 1 reads ordinary bucket runs through idx.
__global__ void k_l1_totals(const uint32_t* __restrict__ off, uint32_t B, uint32_t CH,
                            uint32_t* __restrict__ tot) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    uint32_t s = 0;
    for (uint32_t c = 0; c < CH; ++c)
        s += (off[(size_t)c * (B + 1) + b + 1] - off[(size_t)c * (B + 1) + b] + 1) >> 1;
    tot[b] = s;
}

// PAIR_J consecutive positions of idx per thread (the level's total is
// in1[B]); in1 holds B + 1 run offsets.
__global__ void k_l1_index(const uint32_t* __restrict__ off, const uint32_t* __restrict__ in1,
                           uint32_t B, uint32_t CH, uint32_t* __restrict__ idx) {
    const uint32_t total = in1[B];
    const unsigned long long s0 = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) * PAIR_J;
    if (s0 >= total) return;
    const uint32_t send = (uint32_t)min((unsigned long long)total, s0 + PAIR_J);
    uint32_t lo = 0, hi = B;  // largest b with in1[b] <= s0
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (in1[mid] <= (uint32_t)s0)
            lo = mid;
        else
            hi = mid;
    }
    uint32_t b = lo;
    for (uint32_t s = (uint32_t)s0; s < send; ++s) {
        while (in1[b + 1] <= s) ++b;
        uint32_t p = s - in1[b];
        for (uint32_t c = 0; c < CH; ++c) {
            const uint32_t o = off[(size_t)c * (B + 1) + b];
            const uint32_t cnt = (off[(size_t)c * (B + 1) + b + 1] - o + 1) >> 1;
            if (p < cnt) {
                idx[s] = o + p;
                break;
            }
            p -= cnt;
        }
    }
}

// Lists buckets spanning more than K2 + 1 chunks (list = {count, ids});
// only they go through the fold levels.
__global__ void k_list_big(const uint32_t* __restrict__ offsets, uint32_t B, uint32_t K, int K2,
                           uint32_t cap, uint32_t* __restrict__ list) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= B) return;
    const uint32_t o = offsets[g], c = offsets[g + 1] - o;
    if (c == 0) return;
    const uint32_t t0 = o / K, t1 = (o + c - 1) / K;
    if (t1 - t0 > (uint32_t)K2) {
        const uint32_t slot = atomicAdd(list, 1u);
        if (slot < cap) list[1 + slot] = g;
    }
}

// Group counts of every fold level at once: counts[(level - 2) big_cap + k]
// for listed big bucket k (zero past the list's end).  One exclusive scan
// of the whole array flattens each level's work; level l reads its slice
// relative to the slice's first value.
__global__ void k_fold_counts(const uint32_t* __restrict__ offsets, uint32_t K, int FK, int levels,
                              const uint32_t* __restrict__ big_list, uint32_t big_cap,
                              uint32_t* __restrict__ counts) {
    const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= (size_t)levels * big_cap) return;
    const int level = 2 + (int)(r / big_cap);
    const uint32_t k = (uint32_t)(r % big_cap);
    uint32_t n = 0;
    if (k < min(big_list[0], big_cap)) {
        const uint32_t g = big_list[1 + k];
        const uint32_t o = offsets[g], c = offsets[g + 1] - o;
        uint32_t t0, np;
        fold_sizes(o, c, K, FK, level, t0, np, n);
    }
    counts[r] = n;
}

// ---------------------------------------------------------------------------
// Plans
// ---------------------------------------------------------------------------

static std::mutex g_tune_mu;
static int g_tune[2][3][48];  // [GLV][curve][log2 n]

void msm_tune_set(int curve, int log_n, int c, bool glv) {
    if (curve < 1 || curve > 2 || log_n < 0 || log_n >= 48) return;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[glv ? 1 : 0][curve][log_n] = c;
}

int msm_tune_get(int curve, int log_n, bool glv) {
    if (curve < 1 || curve > 2 || log_n < 0 || log_n >= 48) return 0;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return g_tune[glv ? 1 : 0][curve][log_n];
}

int reference_best_c(size_t n) {
    // (256/c) * (n + 2^c), minimised over c in [4, 12]; first minimum wins.
    int best = 4;
    unsigned long long best_cost = std::numeric_limits<unsigned long long>::max();
    for (int c = 4; c <= 12; ++c) {
        const unsigned long long w = (256 + c - 1) / c;
        const unsigned long long cost = w * ((unsigned long long)n + (1ull << c));
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

static int windows_for(int c) { return (257 + c - 1) / c; }
int msm_windows_for(int c) { return windows_for(c); }

// Live buckets of the top window: its raw digit has 256 - c(W-1) bits plus a
// carry, so its largest magnitude is 2^(256 - c(W-1)).
static uint32_t top_buckets(int c, int W, int scalar_bits = 256) {
    const int bits = scalar_bits - c * (W - 1);
    const uint32_t M = 1u << (c - 1);
    if (bits <= 0) return 1;
    if (bits >= c - 1) return M;
    return 1u << bits;
}

// GLV halves: |k1|, |k2| <= glv_bound(curve), so ceil(bits / c) windows
// cover them, the top window unsigned (its digit is the raw bits plus the
// carry from below, never negated) so nothing carries beyond it.
//   BLS12-381: k1 = k mod lambda, k2 = k div lambda, both at most
//     max(lambda - 1, (r - 1) / lambda) = 0xac45a4010001a402_0000000100000000.
//   BN254: Babai rounding on a reduced lattice basis; both magnitudes at
//     most (|a1| + |a2|) (1/2 + 2^-129) < 0x37a6c124775c2cfecadc035e53799c78.
static unsigned __int128 glv_bound(int curve) {
    if (curve == 2)
        return ((unsigned __int128)0xac45a4010001a402ull << 64) | (unsigned __int128)0x0000000100000000ull;
    return ((unsigned __int128)0x37a6c124775c2cfeull << 64) | (unsigned __int128)0xcadc035e53799c78ull;
}
static int glv_bits(int curve) { return curve == 2 ? 128 : 126; }

// Live buckets of the top window of a GLV half (for c = 4, 8, 16 on
// BLS12-381 its digit exceeds 2^(c-1)).
static uint32_t glv_top_buckets(int curve, int c, int W) {
    const unsigned __int128 bound = glv_bound(curve);
    const int sh = c * (W - 1);
    return (uint32_t)(sh >= 128 ? 0 : (bound >> sh)) + 1u;
}

static int ceil_log2(size_t n) {
    int l = 0;
    while (((size_t)1 << l) < n) ++l;
    return l;
}

MsmPlan make_msm_plan(int curve, size_t n, const MsmOptions& opt) {
    MsmPlan p;
    static const int env_c = [] {
        const char* v = std::getenv("KB200_MSM_C");
        return v && *v ? std::atoi(v) : 0;
    }();
    int c = opt.force_c > 0 ? opt.force_c : env_c;
    if (c <= 0) c = msm_tune_get(curve, ceil_log2(n ? n : 1), false);
    if (c <= 0) {
        // Cost model in accumulation-entry units: one per entry over the
        // windows that canonical (< 2^255) scalars populate, plus ~7 per
        // bucket for the reduction (its two full additions, scan and tree
        // phases; measured on B200 at 2^20-2^22).
        double best = 1e300;
        for (int cc = 4; cc <= 20; ++cc) {
            const double wl = (double)((255 + cc - 1) / cc);
            const double red = wl * (double)n >= PAIRED_ENTRIES ? RED_COST_PAIRED : RED_COST;
            const double cost = wl * (double)n + red * wl * (double)(1u << (cc - 1));
            if (cost < best) {
                best = cost;
                c = cc;
            }
        }
    }
    if (c < 2) c = 2;
    if (c > 22) c = 22;
    p.c = c;
    p.W = windows_for(c);
    p.M = 1u << (c - 1);
    p.M_top = top_buckets(c, p.W);
    return p;
}

MsmPlan make_msm_plan_glv(int curve, size_t n, const MsmOptions& opt) {
    MsmPlan p;
    static const int env_c = [] {
        const char* v = std::getenv("KB200_MSM_GLV_C");
        return v && *v ? std::atoi(v) : 0;
    }();
    const int hb = glv_bits(curve);
    int c = opt.force_c > 0 ? opt.force_c : env_c;
    if (c <= 0) c = msm_tune_get(curve, ceil_log2(n ? n : 1), true);
    if (c <= 0) {
        // 2n points, ceil(hb/c) populated windows of the halves.
        double best = 1e300;
        for (int cc = 4; cc <= 20; ++cc) {
            const double wl = (double)((hb + cc - 1) / cc);
            const double red = wl * 2.0 * (double)n >= PAIRED_ENTRIES ? RED_COST_PAIRED : RED_COST;
            const double cost = wl * 2.0 * (double)n + red * wl * (double)(1u << (cc - 1));
            if (cost < best) {
                best = cost;
                c = cc;
            }
        }
    }
    if (c < 2) c = 2;
    if (c > 22) c = 22;
    p.c = c;
    p.W = (hb + c - 1) / c;
    p.M = 1u << (c - 1);
    p.M_top = glv_top_buckets(curve, c, p.W);
    return p;
}

bool msm_wire_uses_glv(int curve, const MsmOptions& opt) {
    if (opt.shift_c > 0) return false;
    return curve == 1 || (curve == 2 && opt.points_in_g1);
}

class MsmBatchPlan {
   public:
    int curve = 0;
    size_t count = 0;
    std::vector<ItemDesc> items;
    std::vector<WinDesc> wins;
    std::vector<BlkDesc> blks;
    unsigned long long total_scalars = 0, L = 0;
    uint32_t B = 0;
    int K = 64, K2 = 8, FK = 4, levels = 0;
    size_t nchunks = 0, big_cap = 0;
    // Batch-affine pairing levels before the accumulation, and bounds on
    // each level's output length (level l: (len_{l-1} + B) / 2).
    int pair_levels = 0;
    std::vector<unsigned long long> pair_len;
    // Per-chunk first pairing level (single item, host-input pipeline): the
    // sort runs over B_sort = B * chunks keys, chunk-major; chunk_len[c]
    // bounds chunk c's level-0 output slots.
    uint32_t chunks = 1, B_sort = 0, chunk_rows = 0;
    bool red_quad = false;  // stage-1 reduction by quads of lanes (k_reduce_blocks_quad)
    // Tiled ranking (k_rank_tiles): one MSM, windows of at most RANK_TILE_M
    // buckets, at least 2^20 entries.
    bool rank_tiles = false;
    uint32_t rt_G = 0, rt_Q = 0, rt_M = 0;
    std::vector<unsigned long long> chunk_len;
    DevBuf d_items, d_wins, d_blks;
    ~MsmBatchPlan() {
        d_items.release();
        d_wins.release();
        d_blks.release();
    }
};

// SM count of the current device and resident 128-thread accumulation blocks
// per SM for a curve, both cached per device.
static int device_sms() {
    static int cache[64] = {0};
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    int& v = cache[dev & 63];
    if (!v) KB_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    return v;
}
static int acc_occupancy(int curve) {
    static int cache[64][3] = {{0}};
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    int& v = cache[dev & 63][curve == 2 ? 2 : 1];
    if (!v) v = std::max(1, msm_launchers(curve).accumulate_occupancy());
    return v;
}

static void build_plan_host(MsmBatchPlan& P, int curve, const MsmItem* items, size_t count,
                            const MsmOptions& opt) {
    P.curve = curve;
    P.count = count;
    P.items.resize(count);
    size_t max_n = 0, total_live = 0;
    std::vector<MsmPlan> plans(count);
    unsigned long long L = 0, B = 0, tot_sc = 0;
    for (size_t i = 0; i < count; ++i) {
        const size_t n = items[i].n;
        if (n >= (1ull << 31) || items[i].point_off + n >= (1ull << 31))
            throw std::invalid_argument("msm: more than 2^31 points");
        const bool glv = opt.glv && opt.shift_c <= 0;
        if (glv) {
            plans[i] = make_msm_plan_glv(curve, n, opt);
            if (items[i].point_off + n > opt.glv_rows || 2 * opt.glv_rows >= (1ull << 31))
                throw std::invalid_argument("msm: item outside the GLV table");
        } else if (opt.shift_c > 0) {
            MsmOptions o2 = opt;
            o2.force_c = opt.shift_c;
            plans[i] = make_msm_plan(curve, n, o2);
            if (items[i].point_off + n > opt.shift_stride ||
                (unsigned long long)plans[i].W * opt.shift_stride >= (1ull << 31))
                throw std::invalid_argument("msm: item outside the shifted table");
        } else {
            plans[i] = make_msm_plan(curve, n, opt);
        }
        ItemDesc& d = P.items[i];
        d.scalar_off = items[i].scalar_off;
        d.out_index = items[i].out_index == SIZE_MAX ? (uint32_t)i : (uint32_t)items[i].out_index;
        d.n = (uint32_t)n;
        d.point_off = (uint32_t)items[i].point_off;
        d.quirk_c = opt.ref_carry_quirk ? reference_best_c(n) : 0;
        d.c = (uint32_t)plans[i].c;
        d.M = plans[i].M;
        d.W = n ? (uint32_t)plans[i].W : 0u;
        d.glv = glv ? 1u : 0u;
        d.glv_off = glv ? (uint32_t)opt.glv_rows : 0u;
        d.chunk_rows = 0;
        d.chunk_stride = 0;
        const bool shifted = opt.shift_c > 0 && !glv;
        d.row_stride = shifted ? (uint32_t)opt.shift_stride : 0u;
        d.Wr = shifted ? (n ? 1u : 0u) : d.W;
        if (n) total_live += shifted ? d.M : (size_t)(d.W - 1) * d.M + plans[i].M_top;
        // Largest bucket: one entry per point per window feeding it (both GLV
        // halves feed a window's buckets; a shifted table's windows share one
        // bucket range).
        max_n = std::max<size_t>(max_n, n * (glv ? 2 : 1) * (shifted ? d.W : 1));
        d.entry_base = L;
        d.bucket_base = (uint32_t)B;
        L += (unsigned long long)d.W * n * (glv ? 2u : 1u);
        // the GLV top window may hold more than M buckets (unsigned digit)
        B += (glv && d.W) ? (unsigned long long)(d.W - 1) * d.M + std::max(d.M, plans[i].M_top)
                          : (unsigned long long)d.Wr * d.M;
        tot_sc = std::max<unsigned long long>(tot_sc, d.scalar_off + n);
    }
    if (B >= 0xffffffffull || L >= 0xffffffffull)
        throw std::invalid_argument("msm: batch too large for 32-bit bucket/entry ids");
    // Scalars must be laid out in item order for the recode binary search.
    for (size_t i = 1; i < count; ++i)
        if (P.items[i].scalar_off < P.items[i - 1].scalar_off + P.items[i - 1].n)
            throw std::invalid_argument("msm: batch items must be in scalar order");
    P.L = L;
    P.B = (uint32_t)B;
    P.total_scalars = tot_sc;
    // Reduction granularity: buckets per thread S (any integer).  A stage-1
    // block costs 2S serial additions plus a fixed 24 levels of scan and
    // trees, so S is the smallest that gives about one 256-thread block per
    // SM; when that is under 4 buckets per thread (few buckets), two blocks
    // per SM instead.  At most 64 buckets per thread, and every window has
    // at most RED_THREADS stage-1 blocks.  Measured stage-1 times, one block
    // per SM against two: BLS12-381 2^22 (273 K buckets) 1.43 / 1.75 ms,
    // BN254 2^24 1.43 / 1.53 ms; 2^18 (41 K buckets) 1.15 / 0.99 ms.
    // Many buckets (>= 12 per thread at one block per SM, e.g. the 524 K of
    // a BLS12-381 2^22 MSM with 16-bit windows over 256-bit scalars) run two
    // blocks per SM as well: the serial additions then hide each other's
    // latency (stage 1 2.65 -> 2.50 ms there; at 983 K buckets 4.26 -> 3.87
    // ms; at 262 K, 7 per thread, one block stays faster, 2.02 vs 2.18 ms).
    // KB200_MSM_RED_BPS forces the blocks per SM.
    static const int env_red_bps = [] {
        const char* v = std::getenv("KB200_MSM_RED_BPS");
        return v && *v ? std::atoi(v) : 0;
    }();
    const size_t per_sm = (size_t)device_sms() * RED_THREADS;
    size_t s_one = (total_live + per_sm - 1) / per_sm;
    size_t bps = 1;
    if (s_one < 4 || s_one >= 12) bps = 2;
    if (env_red_bps > 0) bps = (size_t)env_red_bps;
    s_one = (total_live + bps * per_sm - 1) / (bps * per_sm);
    // Each window rounds its block count up, so the S that covers the total
    // can still leave a few blocks for a second wave, which costs a whole
    // block's latency (24 levels of scan and trees) for them alone: raise S
    // (at most to twice) until every block fits the first wave (BLS12-381
    // 2^22: S 7 -> 8 takes 305 blocks to 257 against 296 slots).
    auto window_live = [&](size_t i, uint32_t w) -> uint32_t {
        const ItemDesc& d = P.items[i];
        return d.row_stride ? d.M : ((w == d.W - 1) ? plans[i].M_top : d.M);
    };
    auto blocks_for = [&](uint32_t S) {
        size_t nb = 0;
        for (size_t i = 0; i < count; ++i)
            for (uint32_t w = 0; w < P.items[i].Wr; ++w) {
                const size_t Mw = window_live(i, w);
                const size_t Sw = std::max<size_t>(S, (Mw + (size_t)RED_THREADS * RED_THREADS - 1) /
                                                          ((size_t)RED_THREADS * RED_THREADS));
                nb += std::max<size_t>(1, (Mw + RED_THREADS * Sw - 1) / (RED_THREADS * Sw));
            }
        return nb;
    };
    uint32_t S0 = (uint32_t)std::min<size_t>(64, std::max<size_t>(1, s_one));
    const size_t slots = bps * (size_t)device_sms();
    if (blocks_for(S0) > slots)
        for (uint32_t S = S0 + 1; S <= std::min<uint32_t>(64, 2 * S0); ++S)
            if (blocks_for(S) <= slots) {
                S0 = S;
                break;
            }
    // Few buckets (KZG commits up to 2^16, blobs): the reduction is bound by
    // the latency of its serial additions, not by throughput, so it runs one
    // quad of lanes per slot with the quad addition (k_reduce_blocks_quad),
    // RED_QSLOTS slots per block and at most RED_QSLOTS blocks per window.
    // KB200_MSM_RED_QUAD=0/1 forces the choice.
    static const int env_quad = [] {
        const char* v = std::getenv("KB200_MSM_RED_QUAD");
        return v && *v ? std::atoi(v) : -1;
    }();
    P.red_quad = env_quad >= 0 ? env_quad != 0 : total_live <= RED_QUAD_MAX_LIVE;
    for (size_t i = 0; i < count; ++i) {
        ItemDesc& d = P.items[i];
        d.win_base = (uint32_t)P.wins.size();
        for (uint32_t w = 0; w < d.Wr; ++w) {
            WinDesc wd;
            wd.bucket_base = d.bucket_base + w * d.M;
            wd.Mw = window_live(i, w);
            const uint32_t per_block_min =
                (uint32_t)(((size_t)wd.Mw + (size_t)RED_THREADS * RED_THREADS - 1) /
                           ((size_t)RED_THREADS * RED_THREADS));
            if (P.red_quad) {
                constexpr size_t QQ = (size_t)RED_QSLOTS * RED_QSLOTS;
                wd.S = (uint32_t)std::max<size_t>(1, ((size_t)wd.Mw + QQ - 1) / QQ);
                wd.blk = (uint32_t)RED_QSLOTS * wd.S;
            } else {
                wd.S = std::max<uint32_t>(S0, std::max<uint32_t>(1, per_block_min));
                wd.blk = (uint32_t)RED_THREADS * wd.S;
            }
            // at least one block: the window's stage 2 runs in its last block
            wd.nb = std::max<uint32_t>(1, (wd.Mw + wd.blk - 1) / wd.blk);
            wd.shift = d.row_stride ? 0u : d.c * w;
            wd.blk_base = (uint32_t)P.blks.size();
            for (uint32_t b = 0; b < wd.nb; ++b)
                P.blks.push_back(BlkDesc{(uint32_t)P.wins.size(), b});
            P.wins.push_back(wd);
        }
    }
    // Pairing levels: while buckets hold at least PAIR_MIN_RUN entries on
    // average, pairing every run's neighbours in affine coordinates (6
    // products per addition, one inversion per level) beats the mixed XYZZ
    // accumulation (10 products), once a level has enough additions to repay
    // its fixed cost (about ten launches and one inversion on one thread,
    // 0.25 ms against 0.13 ns saved per addition).  Each level's output is bounded by
    // (len + B) / 2 (a run of m gives ceil(m/2)).  KB200_MSM_PAIR_LEVELS or
    // MsmOptions::pair_levels fixes the number of levels instead.
    P.pair_levels = 0;
    P.pair_len.clear();
    {
        static const int env_levels = [] {
            const char* v = std::getenv("KB200_MSM_PAIR_LEVELS");
            return v && *v ? std::atoi(v) : -1;
        }();
        const int fixed = opt.pair_levels >= 0 ? opt.pair_levels : env_levels;
        const int max_levels = fixed >= 0 ? fixed : PAIR_MAX_LEVELS;
        // per-chunk level 0 splits every run into up to CH sub-runs (one more
        // odd remainder each)
        const uint32_t CH = (opt.point_chunks > 1 && count == 1 && P.items[0].n >= (uint32_t)opt.point_chunks)
                                ? (uint32_t)opt.point_chunks
                                : 1u;
        unsigned long long len = L;
        while (P.pair_levels < max_levels && total_live > 0 &&
               (fixed >= 0 || ((double)len >= PAIR_MIN_RUN * (double)total_live &&
                               len / 2 >= PAIR_MIN_SLOTS))) {
            len = (len + B * (P.pair_levels == 0 ? CH : 1u)) / 2;
            P.pair_len.push_back(len);
            ++P.pair_levels;
        }
        L = len;  // entries left for the accumulation (upper bound)
        for (int l = 0; l < P.pair_levels; ++l) max_n = (max_n + 1) / 2;
        P.chunks = P.pair_levels > 0 ? CH : 1u;
        P.B_sort = P.B * P.chunks;
        P.chunk_rows = 0;
        P.chunk_len.clear();
        if (P.chunks > 1) {
            ItemDesc& d = P.items[0];
            const uint32_t S = (d.n + P.chunks - 1) / P.chunks;
            P.chunk_rows = S;
            d.chunk_rows = S;
            d.chunk_stride = P.B;
            if ((unsigned long long)P.B * P.chunks >= 0xffffffffull)
                throw std::invalid_argument("msm: too many chunk-major sort keys");
            const unsigned long long per_row = (unsigned long long)d.W * (d.glv ? 2u : 1u);
            for (uint32_t c = 0; c < P.chunks; ++c) {
                const unsigned long long lo = (unsigned long long)c * S;
                const unsigned long long hi = std::min<unsigned long long>(lo + S, d.n);
                const unsigned long long ent = hi > lo ? (hi - lo) * per_row : 0ull;
                P.chunk_len.push_back((ent + P.B) / 2);
            }
        }
    }
    // Tiled ranking (k_rank_tiles) for one MSM with at least 2^20 entries
    // whose windows fit a tile's shared-memory counters; about one tile per
    // SM and group in every row chunk.
    P.rank_tiles = false;
    if (count == 1 && P.L >= (1ull << 20)) {
        const ItemDesc& d = P.items[0];
        if (d.n && d.entry_base == 0 && d.scalar_off == 0 && !d.row_stride && d.M <= RANK_TILE_M &&
            P.L % d.n == 0) {
            P.rank_tiles = true;
            P.rt_G = (uint32_t)(P.L / d.n);
            P.rt_Q = std::max<uint32_t>(1, ((uint32_t)device_sms() + P.rt_G - 1) / P.rt_G);
            P.rt_M = d.M;
        }
    }
    // Chunk length: long chunks amortise the per-chunk records, but there must
    // be at least two chunks per resident accumulation thread.
    int K = opt.force_K;
    if (K <= 0) {
        const unsigned long long resident =
            (unsigned long long)device_sms() * acc_occupancy(curve) * 128;
        K = 64;
        while (K > 4 && (unsigned long long)K * resident * 2 > L) K >>= 1;
    }
    P.K = K;
    P.K2 = 8;
    P.nchunks = (size_t)((L + (unsigned long long)K - 1) / (unsigned long long)K);
    // A bucket holds at most max_n entries (see above), so spans at most max_n / K + 1
    // chunks; its chunk records fold in ceil(log_FK(span)) levels.  A big
    // bucket spans more than K2 + 1 chunks, so it owns at least K2 interior
    // chunks outright: at most nchunks / K2 buckets can be big.
    const size_t max_span = (max_n + K - 1) / K + 1;
    int lv = 0;
    size_t span = 1;
    while (span < max_span) {
        span *= (size_t)P.FK;
        ++lv;
    }
    P.levels = max_span > (size_t)P.K2 + 1 ? lv : 0;
    P.big_cap = P.nchunks / (size_t)P.K2 + 2;
}

static void upload_plan(MsmBatchPlan* P, cudaStream_t st) {
    P->d_items.reserve(std::max<size_t>(1, P->items.size()) * sizeof(ItemDesc), st);
    P->d_wins.reserve(std::max<size_t>(1, P->wins.size()) * sizeof(WinDesc), st);
    P->d_blks.reserve(std::max<size_t>(1, P->blks.size()) * sizeof(BlkDesc), st);
    if (!P->items.empty())
        KB_CUDA(cudaMemcpyAsync(P->d_items.ptr, P->items.data(), P->items.size() * sizeof(ItemDesc),
                                cudaMemcpyHostToDevice, st));
    if (!P->wins.empty())
        KB_CUDA(cudaMemcpyAsync(P->d_wins.ptr, P->wins.data(), P->wins.size() * sizeof(WinDesc),
                                cudaMemcpyHostToDevice, st));
    if (!P->blks.empty())
        KB_CUDA(cudaMemcpyAsync(P->d_blks.ptr, P->blks.data(), P->blks.size() * sizeof(BlkDesc),
                                cudaMemcpyHostToDevice, st));
}

MsmBatchPlan* msm_batch_plan_create(int curve, const MsmItem* items, size_t count,
                                    const MsmOptions& opt, cudaStream_t st) {
    auto* P = new MsmBatchPlan();
    try {
        build_plan_host(*P, curve, items, count, opt);
        upload_plan(P, st);
        KB_CUDA(cudaStreamSynchronize(st));
    } catch (...) {
        delete P;
        throw;
    }
    return P;
}

void msm_batch_plan_update(MsmBatchPlan* P, const MsmItem* items, size_t count,
                           const MsmOptions& opt, cudaStream_t st) {
    P->items.clear();
    P->wins.clear();
    P->blks.clear();
    build_plan_host(*P, P->curve, items, count, opt);
    upload_plan(P, st);  // stream-ordered after every earlier launch that read it
}

void msm_batch_plan_destroy(MsmBatchPlan* p) { delete p; }
size_t msm_batch_plan_count(const MsmBatchPlan* p) { return p->count; }

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------

constexpr int N_STAGE_EVENTS = 9;

class MsmEngine {
   public:
    int curve = 0;
    DevBuf table, keys, vals, counts, offsets, cursor, sorted, rec_first, rec_last, fold_buf,
        buckets, blk_out, win_out, win_done, l1_idx, chunk_base, scan_tmp, queue, fold_counts, fold_prefix, ranks, pair_off[2],
        pair_rows[2], pair_scratch, pair_cntT, pair_dst, pair_in1;
    std::map<std::tuple<size_t, bool, int, int, int, size_t, bool, size_t, int>, MsmBatchPlan*> single_plans;
    cudaEvent_t ev[N_STAGE_EVENTS] = {};
    bool ev_ready = false, ev_recorded = false;
    // Host-input pipeline (msm_run_host_wire): copy and conversion streams,
    // and events for the start, each point chunk and the finished table.
    // Point chunks of the host pipeline: 4 (measured at 2^22: 2, 3, 4, 6, 8
    // chunks give 36.1, 36.5, 35.8, 36.9, 38.5 ms end to end; each chunk's
    // first pairing level pays its own inversion tree and launches).
    static constexpr int HOST_CHUNKS_MAX = 8;
    static constexpr int HOST_CHUNKS = 4;
    cudaStream_t st_copy = nullptr, st_conv = nullptr, st_sort = nullptr;
    cudaEvent_t ev_start = nullptr, ev_chunk[HOST_CHUNKS_MAX] = {}, ev_conv[HOST_CHUNKS_MAX] = {},
                ev_scal[HOST_CHUNKS_MAX] = {}, ev_sorted[HOST_CHUNKS_MAX] = {}, ev_fork = nullptr;
    void host_streams() {
        if (st_copy) return;
        KB_CUDA(cudaStreamCreateWithFlags(&st_copy, cudaStreamNonBlocking));
        KB_CUDA(cudaStreamCreateWithFlags(&st_conv, cudaStreamNonBlocking));
        KB_CUDA(cudaStreamCreateWithFlags(&st_sort, cudaStreamNonBlocking));
        KB_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        for (auto& c : ev_sorted) KB_CUDA(cudaEventCreateWithFlags(&c, cudaEventDisableTiming));
        KB_CUDA(cudaEventCreateWithFlags(&ev_start, cudaEventDisableTiming));
        for (auto& c : ev_chunk) KB_CUDA(cudaEventCreateWithFlags(&c, cudaEventDisableTiming));
        for (auto& c : ev_conv) KB_CUDA(cudaEventCreateWithFlags(&c, cudaEventDisableTiming));
        for (auto& c : ev_scal) KB_CUDA(cudaEventCreateWithFlags(&c, cudaEventDisableTiming));
    }
    void mark(int i, cudaStream_t st) {
        if (!profiling_enabled()) return;
        if (!ev_ready) {
            for (auto& e : ev) KB_CUDA(cudaEventCreate(&e));
            ev_ready = true;
        }
        KB_CUDA(cudaEventRecord(ev[i], st));
        if (i == N_STAGE_EVENTS - 1) ev_recorded = true;
    }
    ~MsmEngine() {
        for (auto& kv : single_plans) delete kv.second;
        if (ev_ready)
            for (auto& e : ev) cudaEventDestroy(e);
        if (st_copy) {
            cudaStreamDestroy(st_copy);
            cudaStreamDestroy(st_conv);
            cudaEventDestroy(ev_start);
            for (auto& c : ev_chunk) cudaEventDestroy(c);
            for (auto& c : ev_conv) cudaEventDestroy(c);
            for (auto& c : ev_scal) cudaEventDestroy(c);
            cudaStreamDestroy(st_sort);
            cudaEventDestroy(ev_fork);
            for (auto& c : ev_sorted) cudaEventDestroy(c);
        }
        for (DevBuf* b : {&table, &keys, &vals, &counts, &offsets, &cursor, &sorted, &rec_first,
                          &rec_last, &fold_buf, &buckets, &blk_out, &win_out, &win_done, &l1_idx,
                          &chunk_base, &scan_tmp, &queue,
                          &fold_counts, &fold_prefix, &ranks, &pair_off[0], &pair_off[1], &pair_rows[0],
                          &pair_rows[1], &pair_scratch, &pair_cntT, &pair_dst, &pair_in1})
            b->release();
    }
};

int table_words(int curve) { return curve == 2 ? 24 : 16; }

MsmEngine* msm_engine_create(int curve) {
    auto* e = new MsmEngine();
    e->curve = curve;
    return e;
}

void msm_engine_destroy(MsmEngine* e) { delete e; }

// Pairing levels of a batch that holds an item of L entries over B buckets
// (counted for every item: a batch pairs globally): its share of the two
// level row buffers ((L + B) / 2 and (L + 3B) / 4 rows of TW bytes), the
// level offsets and the inversion scratch of the first level.
static size_t pair_item_bytes(size_t TW, size_t L, size_t B) {
    const size_t len0 = (L + B) / 2 + 1, len1 = (L + 3 * B) / 4 + 1;
    return (len0 + len1) * TW + 8 * (B + 1) +
           pair_scratch_words(pair_threads(len0) + 1, (int)(TW / 8)) * 4;
}

// Upper bounds without building a plan (admission control calls these per
// request).  Per item, with its plain-table window plan: keys, vals and the
// sorted list and the ranks (4 B per entry each), three 4 B bucket arrays and the bucket
// accumulators (per bucket), and the reduction blocks of its windows.
size_t msm_item_scratch_bytes(int curve, size_t n) {
    const size_t PW = (size_t)(curve == 2 ? 48 : 32) * 4;
    const MsmPlan p = make_msm_plan(curve, n, MsmOptions());
    const size_t L = (size_t)p.W * n, B = (size_t)p.W * p.M;
    return 16 * L + 12 * (B + 1) + B * PW + (size_t)p.W * (2 * RED_THREADS + 1) * PW +
           (L / 64 + 1) * (3 * PW + 4) +  // chunk records once lists are long (K = 64)
           pair_item_bytes(PW / 2, L, B);
}

// Per batch: the chunk records of short lists (K < 64 keeps at most about two
// chunks per resident accumulation thread) and 1 MiB of descriptors.
size_t msm_batch_fixed_bytes(int curve) {
    const size_t PW = (size_t)(curve == 2 ? 48 : 32) * 4;
    return (size_t)2 * 148 * 8 * 128 * (3 * PW + 4) + ((size_t)1 << 20);
}

size_t msm_scratch_bytes(int curve, const size_t* ns, size_t count) {
    size_t b = msm_batch_fixed_bytes(curve);
    for (size_t i = 0; i < count; ++i) b += msm_item_scratch_bytes(curve, ns[i]);
    return b;
}

void msm_engine_reserve(MsmEngine* e, const MsmBatchPlan* p, cudaStream_t st) {
    const MsmBatchPlan& P = *p;
    const size_t PW = (size_t)msm_launchers(e->curve).point_words;
    const size_t L = std::max<size_t>(1, (size_t)P.L);
    e->keys.reserve(L * 4, st);
    e->vals.reserve(L * 4, st);
    e->sorted.reserve(L * 4, st);
    e->ranks.reserve(L * 4, st);
    const size_t BS = std::max<size_t>(P.B, P.B_sort);
    e->counts.reserve((BS + 1) * 4, st);
    // the host-input pipeline keeps each row chunk's B + 1 offsets apart
    e->offsets.reserve(std::max(BS + 1, (size_t)P.chunks * ((size_t)P.B + 1) + 1) * 4, st);
    e->cursor.reserve((BS + 1) * 4, st);
    const size_t nch = std::max<size_t>(1, P.nchunks);
    e->rec_first.reserve(nch * PW * 4, st);
    e->rec_last.reserve(nch * PW * 4, st);
    if (P.levels >= 1) e->fold_buf.reserve(nch * PW * 4, st);
    e->buckets.reserve(std::max<size_t>(1, (size_t)P.B) * PW * 4, st);
    e->blk_out.reserve(std::max<size_t>(1, P.blks.size()) * 2 * PW * 4, st);
    e->win_out.reserve(std::max<size_t>(1, P.wins.size()) * PW * 4, st);
    e->win_done.reserve(std::max<size_t>(1, P.wins.size()) * 4, st);
    e->scan_tmp.reserve(
        scan_tmp_words(std::max<size_t>(BS, (size_t)std::max(1, P.levels) * P.big_cap) + 1) * 4, st);
    const size_t fold_all = (size_t)std::max(1, P.levels) * P.big_cap;
    e->fold_counts.reserve((fold_all + 1) * 4, st);
    e->fold_prefix.reserve((fold_all + 1) * 4, st);
    e->queue.reserve((P.big_cap + 8) * 4, st);
    if (P.pair_levels > 0) {
        const size_t TW = (size_t)msm_launchers(e->curve).table_words;
        if (P.chunks > 1) {
            e->pair_cntT.reserve((BS + 1) * 4, st);
            e->pair_dst.reserve((BS + 1) * 4, st);
            e->pair_in1.reserve(((size_t)P.B + 1) * 4, st);
            // host-input pipeline: per-chunk first-level offsets, level 1's
            // index, the chunks' running totals
            e->l1_idx.reserve((P.pair_len[0] + 1) * 4, st);
            e->chunk_base.reserve(((size_t)P.chunks + 1) * 4, st);
        }
        for (int k = 0; k < 2 && k < P.pair_levels; ++k) {
            e->pair_off[k].reserve((BS + P.chunks + 1) * 4, st);
            // chunked: the first level writes each sub-run's sums at its own
            // entry positions (up to L rows)
            const unsigned long long rows =
                (k == 0 && P.chunks > 1) ? std::max<unsigned long long>(P.pair_len[0], P.L) : P.pair_len[k];
            e->pair_rows[k].reserve(std::max<unsigned long long>(1, rows) * TW * 4, st);
        }
        e->pair_scratch.reserve(pair_scratch_words(pair_threads(P.pair_len[0]), (int)TW / 2) * 4, st);
    }
}

void msm_engine_launch(MsmEngine* e, const MsmBatchPlan* p, const uint8_t* d_scalars,
                       const uint32_t* d_table, uint8_t* d_out_wire, uint8_t* d_out_comp,
                       cudaStream_t st, const cudaEvent_t* table_ready, int n_ready,
                       const cudaEvent_t* scalars_ready) {
    const MsmBatchPlan& P = *p;
    const MsmLaunchers& K = msm_launchers(e->curve);
    const ItemDesc* items = P.d_items.as<ItemDesc>();
    const uint32_t nitems = (uint32_t)P.count;
    static const bool trace = std::getenv("KB200_SERVE_TRACE") != nullptr;
    auto tt = std::chrono::steady_clock::now();
    auto lap = [&](int where) {
        if (!trace) return;
        const auto t1 = std::chrono::steady_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(t1 - tt).count();
        if (ms > 2.0) std::fprintf(stderr, "[msm] launch step %d: %.3f ms\n", where, ms);
        tt = t1;
    };
    const uint32_t BS = std::max<uint32_t>(P.B, P.B_sort);  // sort keys
    KB_CUDA(cudaMemsetAsync(e->counts.ptr, 0, ((size_t)BS + 1) * 4, st));
    const uint32_t* scal = reinterpret_cast<const uint32_t*>(d_scalars);
    const uint32_t* rec_table = table_ready ? nullptr : d_table;
    // Scalars arriving in row chunks (one MSM; entry slot g * n + j): each
    // chunk's recode and ranking start as soon as it lands.
    const size_t n0 = P.count == 1 ? (size_t)P.items[0].n : 0;
    const bool by_rows = scalars_ready && n_ready > 0 && n0 > 0 && P.L > 0 && P.L % n0 == 0 &&
                         P.items[0].entry_base == 0 && P.items[0].scalar_off == 0;
    // Tiled ranking: row chunks of the scalar arrival (or of the chunk-major
    // keys), tiles per (chunk, group); see k_rank_tiles.
    RankTiles rt{};
    uint32_t rt_chunks = 0;
    if (P.rank_tiles) {
        rt_chunks = by_rows ? (uint32_t)n_ready : (P.chunk_rows ? P.chunks : 1u);
        const ItemDesc& d = P.items[0];
        rt.n = d.n;
        rt.G = P.rt_G;
        rt.TS = (uint32_t)((n0 + rt_chunks - 1) / rt_chunks);
        rt.Q = P.rt_Q;
        rt.R = (rt.TS + rt.Q - 1) / rt.Q;
        rt.M = P.rt_M;
        rt.glv = d.glv;
        rt.bucket_base = d.bucket_base;
        rt.chunk_rows = d.chunk_rows;
        rt.chunk_stride = d.chunk_stride;
        if (d.chunk_rows && d.chunk_rows != rt.TS) rt_chunks = 0;  // tiles must not straddle key chunks
    }
    const bool tiled = rt_chunks > 0;
    const size_t tile_smem = (size_t)rt.M * 4;
    if (tiled) set_smem_attr((const void*)k_rank_tiles, tile_smem);
    // Host-input pipeline with the first pairing level per row chunk: every
    // chunk is sorted (its keys are its own range, chunk-major), scanned from
    // the previous chunk's total and paired as soon as its own scalars and
    // points are resident, instead of after every scalar; level 1 then reads
    // the chunks' sums through an index (k_l1_index).
    const size_t S_rows = n_ready > 0 ? (n0 + n_ready - 1) / n_ready : 0;
    const bool pipelined = by_rows && P.chunks > 1 && P.pair_levels > 0 && table_ready &&
                           n_ready == (int)P.chunks && P.chunk_rows == S_rows &&
                           P.items[0].chunk_stride == P.B;
    if (by_rows) {
        const size_t G = P.L / n0, S = S_rows;
        // pipelined: the chunks' sorts run on a stream of their own, so chunk
        // c + 1 sorts while chunk c pairs
        cudaStream_t ss = st;
        if (pipelined) {
            e->host_streams();
            ss = e->st_sort;
            KB_CUDA(cudaEventRecord(e->ev_fork, st));
            KB_CUDA(cudaStreamWaitEvent(ss, e->ev_fork, 0));
        }
        for (int c = 0; c < n_ready; ++c) {
            const size_t lo = std::min(n0, (size_t)c * S), hi = std::min(n0, lo + S);
            KB_CUDA(cudaStreamWaitEvent(ss, scalars_ready[c], 0));
            if (hi == lo && !pipelined) continue;
            K.recode(items, nitems, lo, hi - lo, scal, rec_table, e->keys.as<uint32_t>(),
                     e->vals.as<uint32_t>(), ss);
            if (tiled) {
                k_rank_tiles<<<dim3(rt.G * rt.Q, 1), RANK_TILE_THREADS, tile_smem, ss>>>(
                    e->keys.as<uint32_t>(), rt, (uint32_t)c, e->counts.as<uint32_t>(),
                    e->ranks.as<uint32_t>());
            } else if (hi > lo) {
                k_rank_rows<<<ceil_div_u(G * (hi - lo), 256), 256, 0, ss>>>(
                    e->keys.as<uint32_t>(), (uint32_t)n0, (uint32_t)G, (uint32_t)lo,
                    (uint32_t)(hi - lo), e->counts.as<uint32_t>(), e->ranks.as<uint32_t>());
            }
            KB_LAUNCH_CHECK();
            if (!pipelined) continue;
            // chunk c: bucket offsets (keys c B .. c B + B - 1, kept at
            // c (B + 1) so that no word is shared with the chunk pairing
            // meanwhile) from the previous chunk's total, scatter, first
            // pairing level
            const uint32_t B = P.B;
            uint32_t* offs = e->offsets.as<uint32_t>() + (size_t)c * (B + 1);
            uint32_t* cnt = e->counts.as<uint32_t>() + (size_t)c * B;
            uint32_t* bases = e->chunk_base.as<uint32_t>();
            exclusive_scan_u32_chained(cnt, offs, B, 0, c ? bases + c : nullptr, bases + c + 1,
                                       e->scan_tmp.as<uint32_t>(), ss);
            if (hi > lo) {
                k_scatter_rows<<<ceil_div_u(G * (hi - lo), 256), 256, 0, ss>>>(
                    e->keys.as<uint32_t>(), e->vals.as<uint32_t>(), e->ranks.as<uint32_t>(),
                    (uint32_t)n0, (uint32_t)G, (uint32_t)lo, (uint32_t)(hi - lo),
                    e->offsets.as<uint32_t>(), (uint32_t)c, e->sorted.as<uint32_t>());
                KB_LAUNCH_CHECK();
            }
            uint32_t* out0 = e->pair_off[0].as<uint32_t>() + (size_t)c * (B + 1);
            k_pair_counts<<<ceil_div_u(B, 256), 256, 0, ss>>>(offs, B, cnt);
            KB_LAUNCH_CHECK();
            exclusive_scan_u32(cnt, out0, B, 0, e->scan_tmp.as<uint32_t>(), ss);
            KB_CUDA(cudaEventRecord(e->ev_sorted[c], ss));
            KB_CUDA(cudaStreamWaitEvent(st, e->ev_sorted[c], 0));
            KB_CUDA(cudaStreamWaitEvent(st, table_ready[c], 0));
            PairArgs pa;
            pa.in_off = offs;
            pa.out_off = out0;
            pa.B = B;
            pa.sorted = e->sorted.as<uint32_t>();
            pa.src = d_table;
            pa.dst = e->pair_rows[0].as<uint32_t>();
            pa.dst_off = offs;  // a sub-run's sums at its own entry positions
            K.pair_level(pa, pair_threads(P.chunk_len[c]), e->pair_scratch.as<uint32_t>(), st);
        }
    } else if (P.L > 0) {
        if (scalars_ready && n_ready > 0) KB_CUDA(cudaStreamWaitEvent(st, scalars_ready[n_ready - 1], 0));
        K.recode(items, nitems, 0, P.total_scalars, scal, rec_table, e->keys.as<uint32_t>(),
                 e->vals.as<uint32_t>(), st);
        if (tiled) {
            k_rank_tiles<<<dim3(rt.G * rt.Q, rt_chunks), RANK_TILE_THREADS, tile_smem, st>>>(
                e->keys.as<uint32_t>(), rt, 0u, e->counts.as<uint32_t>(), e->ranks.as<uint32_t>());
        } else {
            k_rank<<<ceil_div_u(P.L, 256), 256, 0, st>>>(e->keys.as<uint32_t>(), P.L,
                                                        e->counts.as<uint32_t>(),
                                                        e->ranks.as<uint32_t>());
        }
        KB_LAUNCH_CHECK();
    }
    e->mark(2, st);
    lap(2);
    if (!pipelined)
        exclusive_scan_u32(e->counts.as<uint32_t>(), e->offsets.as<uint32_t>(), BS, 0,
                           e->scan_tmp.as<uint32_t>(), st);
    if (P.L > 0 && !pipelined) {
        k_scatter<<<ceil_div_u(P.L, 256), 256, 0, st>>>(
            e->keys.as<uint32_t>(), e->vals.as<uint32_t>(), e->ranks.as<uint32_t>(), P.L,
            e->offsets.as<uint32_t>(), e->sorted.as<uint32_t>());
        KB_LAUNCH_CHECK();
    }
    e->mark(3, st);
    lap(3);
    const bool per_chunk = P.chunks > 1 && table_ready && n_ready == (int)P.chunks && P.L > 0;
    if (table_ready && n_ready > 0 && !per_chunk)
        KB_CUDA(cudaStreamWaitEvent(st, table_ready[n_ready - 1], 0));
    if (pipelined) {
        // level 1's runs: bucket by bucket over the chunks' first-level sums
        const uint32_t CH = P.chunks, B = P.B;
        k_l1_totals<<<ceil_div_u(B, 256), 256, 0, st>>>(e->offsets.as<uint32_t>(), B, CH,
                                                       e->counts.as<uint32_t>());
        KB_LAUNCH_CHECK();
        exclusive_scan_u32(e->counts.as<uint32_t>(), e->pair_in1.as<uint32_t>(), B, 0,
                           e->scan_tmp.as<uint32_t>(), st);
        k_l1_index<<<ceil_div_u(pair_threads(P.pair_len[0]), 256), 256, 0, st>>>(
            e->offsets.as<uint32_t>(), e->pair_in1.as<uint32_t>(), B, CH, e->l1_idx.as<uint32_t>());
        KB_LAUNCH_CHECK();
    }
    // Pairing levels: the sorted runs shrink to about half per level, the
    // accumulation then reads the last level's rows directly.
    const uint32_t* off = e->offsets.as<uint32_t>();
    const uint32_t* acc_sorted = e->sorted.as<uint32_t>();
    const uint32_t* acc_table = d_table;
    int l0 = 0;
    if (pipelined) {
        off = e->pair_in1.as<uint32_t>();
        acc_sorted = e->l1_idx.as<uint32_t>();
        acc_table = e->pair_rows[0].as<uint32_t>();
        l0 = 1;
    } else if (P.chunks > 1 && P.pair_levels > 0 && P.L > 0) {
        // Level 0 per chunk of points: sub-run (c, b) pairs only the points of
        // chunk c, so chunk c runs as soon as its rows exist; its sums land
        // at bucket-major rows, so level 1 reads ordinary bucket runs.
        const uint32_t CH = P.chunks, B = P.B;
        uint32_t* out_off = e->pair_off[0].as<uint32_t>();
        k_pair_counts<<<ceil_div_u(BS, 256), 256, 0, st>>>(off, BS, e->counts.as<uint32_t>());
        KB_LAUNCH_CHECK();
        exclusive_scan_u32(e->counts.as<uint32_t>(), out_off, BS, 0, e->scan_tmp.as<uint32_t>(), st);
        k_transpose_counts<<<ceil_div_u(BS, 256), 256, 0, st>>>(e->counts.as<uint32_t>(), B, CH,
                                                               e->pair_cntT.as<uint32_t>());
        KB_LAUNCH_CHECK();
        uint32_t* scanT = e->cursor.as<uint32_t>();  // free once the scatter is done
        exclusive_scan_u32(e->pair_cntT.as<uint32_t>(), scanT, BS, 0, e->scan_tmp.as<uint32_t>(), st);
        k_chunk_offsets<<<ceil_div_u((size_t)BS + 1, 256), 256, 0, st>>>(
            scanT, B, CH, e->pair_dst.as<uint32_t>(), e->pair_in1.as<uint32_t>());
        KB_LAUNCH_CHECK();
        for (uint32_t c = 0; c < CH; ++c) {
            if (per_chunk) KB_CUDA(cudaStreamWaitEvent(st, table_ready[c], 0));
            PairArgs pa;
            pa.in_off = off + (size_t)c * B;
            pa.out_off = out_off + (size_t)c * B;
            pa.B = B;
            pa.sorted = acc_sorted;
            pa.src = acc_table;
            pa.dst = e->pair_rows[0].as<uint32_t>();
            pa.dst_off = e->pair_dst.as<uint32_t>() + (size_t)c * B;
            K.pair_level(pa, pair_threads(P.chunk_len[c]), e->pair_scratch.as<uint32_t>(), st);
        }
        off = e->pair_in1.as<uint32_t>();
        acc_sorted = nullptr;
        acc_table = e->pair_rows[0].as<uint32_t>();
        l0 = 1;
    }
    for (int l = l0; l < P.pair_levels && P.L > 0; ++l) {
        uint32_t* out_off = e->pair_off[l & 1].as<uint32_t>();
        k_pair_counts<<<ceil_div_u(P.B, 256), 256, 0, st>>>(off, P.B, e->counts.as<uint32_t>());
        KB_LAUNCH_CHECK();
        exclusive_scan_u32(e->counts.as<uint32_t>(), out_off, P.B, 0, e->scan_tmp.as<uint32_t>(), st);
        PairArgs pa;
        pa.in_off = off;
        pa.out_off = out_off;
        pa.B = P.B;
        pa.sorted = acc_sorted;
        pa.src = acc_table;
        pa.dst = e->pair_rows[l & 1].as<uint32_t>();
        pa.dst_off = nullptr;
        const unsigned long long slots = P.pair_len[l];
        K.pair_level(pa, pair_threads(slots), e->pair_scratch.as<uint32_t>(), st);
        off = out_off;
        acc_sorted = nullptr;
        acc_table = e->pair_rows[l & 1].as<uint32_t>();
    }
    KB_CUDA(cudaMemsetAsync(e->queue.ptr, 0, 8, st));  // work counter, big-bucket count
    uint32_t* big_list = e->queue.as<uint32_t>() + 1;
    if (P.B > 0 && P.levels >= 1) {
        k_list_big<<<ceil_div_u(P.B, 256), 256, 0, st>>>(off, P.B,
                                                        (uint32_t)P.K, P.K2, (uint32_t)P.big_cap,
                                                        big_list);
        KB_LAUNCH_CHECK();
    }
    e->mark(4, st);
    lap(4);

    AccArgs acc;
    acc.sorted = acc_sorted;
    acc.offsets = off;
    acc.B = P.B;
    acc.K = (uint32_t)P.K;
    acc.table = acc_table;
    acc.rec_first = e->rec_first.as<uint32_t>();
    acc.rec_last = e->rec_last.as<uint32_t>();
    acc.buckets = e->buckets.as<uint32_t>();
    acc.queue = e->queue.as<uint32_t>();
    if (P.L > 0) {
        const size_t units = (P.nchunks + 127) / 128;
        const unsigned grid =
            (unsigned)std::min<size_t>(units, (size_t)device_sms() * acc_occupancy(e->curve));
        K.accumulate(acc, std::max(1u, grid), st);
    }
    e->mark(5, st);
    lap(5);

    if (P.levels >= 1 && P.L > 0) {
        FoldArgs fa;
        fa.offsets = off;
        fa.B = P.B;
        fa.K = (uint32_t)P.K;
        fa.K2 = P.K2;
        fa.FK = P.FK;
        fa.big_list = big_list;
        fa.big_cap = (uint32_t)P.big_cap;
        fa.prefix = e->fold_prefix.as<uint32_t>();
        fa.rec_first = e->rec_first.as<uint32_t>();
        uint32_t* in = e->rec_first.as<uint32_t>();
        uint32_t* out = e->fold_buf.as<uint32_t>();
        const size_t all = (size_t)P.levels * P.big_cap;
        k_fold_counts<<<ceil_div_u(all, 256), 256, 0, st>>>(off, (uint32_t)P.K, P.FK, P.levels, big_list,
                                                           (uint32_t)P.big_cap,
                                                           e->fold_counts.as<uint32_t>());
        KB_LAUNCH_CHECK();
        exclusive_scan_u32(e->fold_counts.as<uint32_t>(), e->fold_prefix.as<uint32_t>(), all, 0,
                           e->scan_tmp.as<uint32_t>(), st);
        for (int l = 2; l <= P.levels + 1; ++l) {
            fa.prefix = e->fold_prefix.as<uint32_t>() + (size_t)(l - 2) * P.big_cap;
            K.fold(fa, l, in, out, (unsigned)device_sms() * 8, st);
            std::swap(in, out);
        }
    }
    e->mark(6, st);
    lap(6);

    RedArgs ra;
    ra.offsets = off;
    ra.B = P.B;
    ra.buckets = e->buckets.as<uint32_t>();
    ra.rec_first = e->rec_first.as<uint32_t>();
    ra.rec_last = e->rec_last.as<uint32_t>();
    ra.K = (uint32_t)P.K;
    ra.K2 = P.K2;
    ra.wins = P.d_wins.as<WinDesc>();
    ra.blks = P.d_blks.as<BlkDesc>();
    ra.blk_out = e->blk_out.as<uint32_t>();
    ra.win_out = e->win_out.as<uint32_t>();
    ra.win_done = e->win_done.as<uint32_t>();
    // one launch: each window's stage 2 runs in the block that finishes it
    KB_CUDA(cudaMemsetAsync(ra.win_done, 0, P.wins.size() * 4, st));
    if (P.red_quad)
        K.reduce_blocks_quad(ra, (unsigned)P.blks.size(), st);
    else
        K.reduce_blocks(ra, (unsigned)P.blks.size(), st);
    e->mark(7, st);
    lap(7);
    K.combine(items, nitems, e->win_out.as<uint32_t>(), d_out_wire, d_out_comp, st);
    e->mark(8, st);
    lap(8);
}

static MsmBatchPlan* single_plan(MsmEngine* e, size_t n, const MsmOptions& opt, cudaStream_t st) {
    auto key = std::make_tuple(n, opt.ref_carry_quirk, opt.force_c, opt.force_K, opt.shift_c,
                               opt.shift_stride, opt.glv, opt.glv_rows, opt.point_chunks);
    auto it = e->single_plans.find(key);
    if (it != e->single_plans.end()) return it->second;
    MsmItem item{0, n, 0};
    MsmBatchPlan* p = msm_batch_plan_create(e->curve, &item, 1, opt, st);
    if (e->single_plans.size() > 64) {
        KB_CUDA(cudaStreamSynchronize(st));
        for (auto& kv : e->single_plans) delete kv.second;
        e->single_plans.clear();
    }
    e->single_plans[key] = p;
    return p;
}

void msm_run_table(MsmEngine* e, const uint8_t* d_scalars, const uint32_t* d_table, size_t n,
                   uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t st,
                   const MsmOptions& opt) {
    MsmBatchPlan* p = single_plan(e, n, opt, st);
    msm_engine_reserve(e, p, st);
    e->mark(0, st);
    e->mark(1, st);
    msm_engine_launch(e, p, d_scalars, d_table, d_out_wire, d_out_comp, st);
}

void msm_run_wire(MsmEngine* e, const uint8_t* d_scalars, const uint8_t* d_points, size_t n,
                  uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t st,
                  const MsmOptions& opt) {
    // GLV split (the table gains the phi(P) rows) where phi(P) = [lambda]P
    // holds for every input point: always on BN254, and on BLS12-381 when
    // the caller vouches that the points lie in G1.
    MsmOptions o2 = opt;
    const bool glv = msm_wire_uses_glv(e->curve, opt);
    if (glv) {
        o2.glv = true;
        o2.glv_rows = n;
    }
    MsmBatchPlan* p = single_plan(e, n, o2, st);
    msm_engine_reserve(e, p, st);
    const MsmLaunchers& K = msm_launchers(e->curve);
    e->table.reserve(std::max<size_t>(1, n) * (glv ? 2 : 1) * (size_t)K.table_words * 4, st);
    e->mark(0, st);
    K.wire_to_table(d_points, e->table.as<uint32_t>(), n, glv ? n : 0, st);
    e->mark(1, st);
    msm_engine_launch(e, p, d_scalars, e->table.as<uint32_t>(), d_out_wire, d_out_comp, st);
}

void msm_run_host_wire(MsmEngine* e, const uint8_t* h_scalars, const uint8_t* h_points, size_t n,
                       uint8_t* d_scalars, uint8_t* d_points, uint8_t* d_out_wire, cudaStream_t st,
                       const MsmOptions& opt) {
    MsmOptions o2 = opt;
    const bool glv = msm_wire_uses_glv(e->curve, opt);
    if (glv) {
        o2.glv = true;
        o2.glv_rows = n;
    }
    // KB200_MSM_HOST_CHUNKS: point chunks of the host pipeline (1 .. HOST_CHUNKS_MAX)
    static const int env_chunks = [] {
        const char* v = std::getenv("KB200_MSM_HOST_CHUNKS");
        return v && *v ? std::atoi(v) : 0;
    }();
    size_t chunks = n >= ((size_t)1 << 16) ? (size_t)MsmEngine::HOST_CHUNKS : 1;
    if (env_chunks > 0) chunks = std::min<size_t>((size_t)env_chunks, (size_t)MsmEngine::HOST_CHUNKS_MAX);
    o2.point_chunks = (int)chunks;
    MsmBatchPlan* p = single_plan(e, n, o2, st);
    msm_engine_reserve(e, p, st);
    const MsmLaunchers& K = msm_launchers(e->curve);
    const size_t TW = (size_t)K.table_words, WB = (size_t)K.wire_bytes;
    e->table.reserve(std::max<size_t>(1, n) * (glv ? 2 : 1) * TW * 4, st);
    e->host_streams();
    uint32_t* table = e->table.as<uint32_t>();
    // The side streams start after everything already queued on st (the
    // staging buffers may still be read by an earlier call).
    KB_CUDA(cudaEventRecord(e->ev_start, st));
    KB_CUDA(cudaStreamWaitEvent(e->st_copy, e->ev_start, 0));
    KB_CUDA(cudaStreamWaitEvent(e->st_conv, e->ev_start, 0));
    // chunk c = rows [c S, (c + 1) S), S = ceil(n / chunks): the rows the
    // plan's chunk-major sort keys (when it pairs per chunk) assign to c.
    // One copy stream.  When the plan pairs per chunk, chunk by chunk (its
    // scalars, then its points): each chunk is sorted and paired once both
    // are resident.  Otherwise all scalars first (the sort needs every key
    // before the first pairing level), each scalar chunk recoded and ranked
    // as it lands, then the points.
    const size_t S = (n + chunks - 1) / chunks;
    const bool interleave = p->chunks == chunks && p->pair_levels > 0 && chunks > 1;
    auto copy_scalars = [&](size_t c) {
        const size_t lo = std::min(n, c * S), hi = std::min(n, lo + S);
        if (hi > lo) {
            KB_CUDA(cudaMemcpyAsync(d_scalars + lo * 32, h_scalars + lo * 32, (hi - lo) * 32,
                                    cudaMemcpyHostToDevice, e->st_copy));
        }
        KB_CUDA(cudaEventRecord(e->ev_scal[c], e->st_copy));
    };
    auto copy_points = [&](size_t c) {
        const size_t lo = std::min(n, c * S), hi = std::min(n, lo + S);
        if (hi > lo) {
            KB_CUDA(cudaMemcpyAsync(d_points + lo * WB, h_points + lo * WB, (hi - lo) * WB,
                                    cudaMemcpyHostToDevice, e->st_copy));
        }
        KB_CUDA(cudaEventRecord(e->ev_chunk[c], e->st_copy));
        KB_CUDA(cudaStreamWaitEvent(e->st_conv, e->ev_chunk[c], 0));
        K.wire_to_table(d_points + lo * WB, table + lo * TW, hi - lo, glv ? n : 0, e->st_conv);
        KB_CUDA(cudaEventRecord(e->ev_conv[c], e->st_conv));
    };
    if (interleave) {
        for (size_t c = 0; c < chunks; ++c) {
            copy_scalars(c);
            copy_points(c);
        }
    } else {
        for (size_t c = 0; c < chunks; ++c) copy_scalars(c);
        for (size_t c = 0; c < chunks; ++c) copy_points(c);
    }
    e->mark(0, st);
    e->mark(1, st);
    msm_engine_launch(e, p, d_scalars, table, d_out_wire, nullptr, st, e->ev_conv, (int)chunks,
                      e->ev_scal);
}

void points_wire_to_table(int curve, const uint8_t* d_wire, uint32_t* d_table, size_t n,
                          cudaStream_t st) {
    msm_launchers(curve).wire_to_table(d_wire, d_table, n, 0, st);
}

void points_table_to_wire(int curve, const uint32_t* d_table, uint8_t* d_wire, size_t n,
                          cudaStream_t st) {
    msm_launchers(curve).table_to_wire(d_table, d_wire, n, st);
}

int msm_stage_ms(MsmEngine* e, float* out, int max) {
    if (!e->ev_recorded) return 0;
    KB_CUDA(cudaEventSynchronize(e->ev[N_STAGE_EVENTS - 1]));
    int k = 0;
    for (int i = 0; i + 1 < N_STAGE_EVENTS && k < max; ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e->ev[i], e->ev[i + 1]) != cudaSuccess) {
            cudaGetLastError();
            ms = -1.f;
        }
        out[k++] = ms;
    }
    return k;
}

}  // namespace kb200
