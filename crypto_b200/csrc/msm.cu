// G1 Pippenger MSM kernels and host driver.  See msm.cuh for the pipeline.
#include "curve.cuh"
#include "msm.cuh"
#include "runtime.cuh"

#include <algorithm>
#include <limits>

namespace kb200 {

constexpr uint32_t SENTINEL = 0xffffffffu;

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------

int reference_best_c(size_t n) {
    // (256/c) * (n + 2^c), minimised over c in [4, 12]; first minimum wins.
    int best = 4;
    unsigned long long best_cost = std::numeric_limits<unsigned long long>::max();
    for (int c = 4; c <= 12; ++c) {
        unsigned long long w = (256 + c - 1) / c;
        unsigned long long cost = w * ((unsigned long long)n + (1ull << c));
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

static int windows_for(int c) { return (257 + c - 1) / c; }

MsmPlan make_msm_plan(int curve, size_t n, const MsmOptions& opt) {
    (void)curve;
    MsmPlan p;
    int c = opt.force_c;
    if (c <= 0) {
        // Cost model: each entry is one mixed addition; each bucket costs
        // about four additions' worth in the reduction.
        double best = 1e300;
        for (int cc = 4; cc <= 20; ++cc) {
            double cost = (double)windows_for(cc) * ((double)n + 4.0 * (double)(1u << (cc - 1)));
            if (cost < best) {
                best = cost;
                c = cc;
            }
        }
    }
    p.c = c;
    p.W = windows_for(c);
    p.M = 1u << (c - 1);
    p.B = (uint32_t)p.W * p.M;
    const size_t L = n * (size_t)p.W;
    int K = opt.force_K;
    if (K <= 0) {
        if (L >= (1u << 24))
            K = 32;
        else if (L >= (1u << 22))
            K = 16;
        else if (L >= (1u << 20))
            K = 8;
        else
            K = 4;
    }
    p.K = K;
    p.K2 = 8;
    // Worst case a bucket holds n entries (one digit per scalar per window).
    size_t max_seg = (n + K - 1) / K;
    int lv = 0;
    size_t span = 1;
    while (span < max_seg) {
        span *= (size_t)p.K2;
        ++lv;
    }
    p.levels = lv;
    p.S = p.M >= 4096 ? 8 : 4;
    if ((uint32_t)p.S > p.M) p.S = (int)p.M;
    p.G = p.M / (uint32_t)p.S;
    p.seg_cap = L / (size_t)K + (size_t)p.B + 1;
    return p;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

template <class C>
__global__ void k_wire_to_table(const uint8_t* __restrict__ wire, uint32_t* __restrict__ table,
                                size_t n) {
    using F = typename C::F;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    wire_to_table<C>(table + i * 2 * F::N, wire + i * C::WIRE);
}

template <class C>
__global__ void k_table_to_wire(const uint32_t* __restrict__ table, uint8_t* __restrict__ wire,
                                size_t n) {
    using F = typename C::F;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t* t = table + i * 2 * F::N;
    uint8_t* o = wire + i * C::WIRE;
    if (aff_is_inf_words<F>(t)) {
        for (int k = 0; k < C::WIRE; ++k) o[k] = 0;
        return;
    }
    Affine<F> a;
    aff_load(a, t);
    Fe<F> x, y;
    fe_from_mont(x, a.x);
    fe_from_mont(y, a.y);
    fe_to_be_bytes(o, x);
    fe_to_be_bytes(o + F::BYTES, y);
}

// Signed-digit recoding.  Entry (w, i) lives at w * n + i.
// quirk_c: 0, or the reference window size (4 or 8) whose dropped top carry
// is reproduced by negating (s, P) -> (2^256 - s, -P) for s above the
// carry threshold 0x8888...88 (c = 4) or 0x8080...80 (c = 8).
template <class C>
__global__ void k_recode(const uint32_t* __restrict__ scalars, const uint32_t* __restrict__ table,
                         size_t n, int c, int W, uint32_t M, int quirk_c,
                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    using F = typename C::F;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool inf = aff_is_inf_words<F>(table + i * 2 * F::N);
    uint32_t s[8];
    const uint4* sp = reinterpret_cast<const uint4*>(scalars + i * 8);
    uint4 a = sp[0], b = sp[1];
    s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
    s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
    uint32_t neg = 0;
    if (quirk_c == 4 || quirk_c == 8) {
        const uint32_t t = quirk_c == 4 ? 0x88888888u : 0x80808080u;
        // s > t repeated across all words?
        int gt = 0;
#pragma unroll
        for (int k = 7; k >= 0; --k) {
            if (gt == 0) {
                if (s[k] > t) gt = 1;
                else if (s[k] < t) gt = -1;
            }
        }
        if (gt == 1) {
            // s <- 2^256 - s
            uint32_t carry = 1;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                uint64_t v = (uint64_t)(~s[k]) + carry;
                s[k] = (uint32_t)v;
                carry = (uint32_t)(v >> 32);
            }
            neg = 1;
        }
    }
    const uint32_t mask = (1u << c) - 1u;
    uint32_t carry = 0;
    for (int w = 0; w < W; ++w) {
        const int off = w * c;
        const int wd = off >> 5, sh = off & 31;
        uint32_t raw = 0;
        if (wd < 8) {
            uint64_t lo = s[wd];
            uint64_t hi = (wd + 1 < 8) ? s[wd + 1] : 0;
            raw = (uint32_t)(((hi << 32) | lo) >> sh) & mask;
        }
        uint32_t d = raw + carry;
        uint32_t sign = 0;
        if (d > M) {
            d = (1u << c) - d;  // |d - 2^c|
            sign = 1;
            carry = 1;
        } else {
            carry = 0;
        }
        const size_t slot = (size_t)w * n + i;
        if (d == 0 || inf) {
            keys[slot] = SENTINEL;
        } else {
            keys[slot] = (uint32_t)w * M + (d - 1);
            vals[slot] = (uint32_t)i | ((sign ^ neg) << 31);
        }
    }
}

__global__ void k_histogram(const uint32_t* __restrict__ keys, size_t total,
                            uint32_t* __restrict__ counts) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const uint32_t key = keys[t];
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, key);
    const int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader && key != SENTINEL)
        atomicAdd(&counts[key], (uint32_t)__popc(peers));
}

__global__ void k_scatter(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                          size_t total, uint32_t* __restrict__ cursor,
                          uint32_t* __restrict__ sorted) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const uint32_t key = keys[t];
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader && key != SENTINEL) base = atomicAdd(&cursor[key], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    if (key == SENTINEL) return;
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    sorted[base + rank] = vals[t];
}

// Largest b in [0, B) with segoff[b] <= s (segoff non-decreasing, segoff[0] = 0).
__device__ __forceinline__ uint32_t find_bucket(const uint32_t* segoff, uint32_t B, uint32_t s) {
    uint32_t lo = 0, hi = B;  // invariant: segoff[lo] <= s < segoff[hi] (segoff[B] = total)
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (segoff[mid] <= s)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

template <class F>
__device__ __forceinline__ void load_table_point(Affine<F>& a, const uint32_t* table, uint32_t idx) {
    const uint4* src = reinterpret_cast<const uint4*>(table + (size_t)idx * 2 * F::N);
    uint32_t w[2 * F::N];
#pragma unroll
    for (int k = 0; k < F::N / 2; ++k) {
        uint4 v = src[k];
        w[4 * k] = v.x;
        w[4 * k + 1] = v.y;
        w[4 * k + 2] = v.z;
        w[4 * k + 3] = v.w;
    }
    aff_load(a, w);
}

// Level 1: thread s sums segment s of the sorted entries.
template <class C>
__global__ void __launch_bounds__(128) k_accumulate(
    const uint32_t* __restrict__ sorted, const uint32_t* __restrict__ offsets,
    const uint32_t* __restrict__ segoff, uint32_t B, const uint32_t* __restrict__ table, int K,
    size_t seg_cap, uint32_t* __restrict__ partial, uint32_t* __restrict__ bid,
    uint32_t* __restrict__ buckets) {
    using F = typename C::F;
    size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= seg_cap) return;
    const uint32_t total = segoff[B];
    if (s >= total) return;
    const uint32_t b = find_bucket(segoff, B, (uint32_t)s);
    const uint32_t q = (uint32_t)s - segoff[b];
    const uint32_t nseg = segoff[b + 1] - segoff[b];
    const uint32_t start = offsets[b] + q * (uint32_t)K;
    const uint32_t end = min(start + (uint32_t)K, offsets[b + 1]);
    Xyzz<F> acc;
    xyzz_set_inf(acc);
    for (uint32_t e = start; e < end; ++e) {
        const uint32_t v = sorted[e];
        Affine<F> a;
        load_table_point<F>(a, table, v & 0x7fffffffu);
        if (v >> 31) fe_neg(a.y, a.y);
        xyzz_add_affine(acc, a);
    }
    bid[s] = b;
    if (nseg == 1)
        xyzz_store(buckets + (size_t)b * 4 * F::N, acc);
    else
        xyzz_store(partial + s * 4 * F::N, acc);
}

// Level l >= 2: fold partial sums K2 at a time.
template <class C>
__global__ void __launch_bounds__(128) k_fold(int level, const uint32_t* __restrict__ bid,
                                              const uint32_t* __restrict__ segoff, uint32_t B,
                                              int K2, size_t seg_cap,
                                              const uint32_t* __restrict__ in,
                                              uint32_t* __restrict__ out,
                                              uint32_t* __restrict__ buckets) {
    using F = typename C::F;
    size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= seg_cap) return;
    const uint32_t total = segoff[B];
    if (s >= total) return;
    const uint32_t b = bid[s];
    const uint32_t base = segoff[b];
    const uint32_t nseg = segoff[b + 1] - base;
    const uint32_t q = (uint32_t)s - base;
    uint32_t n_prev = nseg;
    for (int l = 2; l < level; ++l) n_prev = (n_prev + K2 - 1) / K2;
    if (n_prev <= 1) return;
    const uint32_t n_cur = (n_prev + K2 - 1) / K2;
    if (q >= n_cur) return;
    const uint32_t lo = q * (uint32_t)K2, hi = min(lo + (uint32_t)K2, n_prev);
    Xyzz<F> acc, t;
    xyzz_load(acc, in + (size_t)(base + lo) * 4 * F::N);
    for (uint32_t j = lo + 1; j < hi; ++j) {
        xyzz_load(t, in + (size_t)(base + j) * 4 * F::N);
        xyzz_add(acc, t);
    }
    if (n_cur == 1)
        xyzz_store(buckets + (size_t)b * 4 * F::N, acc);
    else
        xyzz_store(out + (size_t)(base + q) * 4 * F::N, acc);
}

// Reduction groups: thread (w, g) returns sum_{k in group} (k+1) * B[w][k].
template <class C>
__global__ void __launch_bounds__(128) k_reduce_groups(const uint32_t* __restrict__ buckets,
                                                       int W, uint32_t M, int S, uint32_t G,
                                                       uint32_t* __restrict__ groups) {
    using F = typename C::F;
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)W * G) return;
    const uint32_t w = (uint32_t)(t / G), g = (uint32_t)(t % G);
    const uint32_t lo = g * (uint32_t)S;
    Xyzz<F> R, T, Bk;
    xyzz_set_inf(R);
    xyzz_set_inf(T);
    for (int k = S - 1; k >= 0; --k) {
        xyzz_load(Bk, buckets + ((size_t)w * M + lo + (uint32_t)k) * 4 * F::N);
        xyzz_add(R, Bk);
        xyzz_add(T, R);
    }
    if (lo != 0) {
        // T += lo * R, by double-and-add over the bits of lo.
        Xyzz<F> acc;
        xyzz_set_inf(acc);
        const int top = 31 - __clz(lo);
        for (int bit = top; bit >= 0; --bit) {
            xyzz_dbl(acc, acc);
            if ((lo >> bit) & 1u) xyzz_add(acc, R);
        }
        xyzz_add(T, acc);
    }
    xyzz_store(groups + t * 4 * F::N, T);
}

template <class F>
__device__ __forceinline__ void xyzz_shfl_down(Xyzz<F>& o, const Xyzz<F>& p, int d) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) {
        o.X.v[i] = __shfl_down_sync(0xffffffffu, p.X.v[i], d);
        o.Y.v[i] = __shfl_down_sync(0xffffffffu, p.Y.v[i], d);
        o.ZZ.v[i] = __shfl_down_sync(0xffffffffu, p.ZZ.v[i], d);
        o.ZZZ.v[i] = __shfl_down_sync(0xffffffffu, p.ZZZ.v[i], d);
    }
}

// One block per window: sum of its G group results.
template <class C>
__global__ void __launch_bounds__(256) k_window_sums(const uint32_t* __restrict__ groups,
                                                     uint32_t G, uint32_t* __restrict__ wins) {
    using F = typename C::F;
    __shared__ uint32_t sm[8][4 * F::N];
    const uint32_t w = blockIdx.x;
    Xyzz<F> acc, t;
    xyzz_set_inf(acc);
    for (uint32_t j = threadIdx.x; j < G; j += blockDim.x) {
        xyzz_load(t, groups + ((size_t)w * G + j) * 4 * F::N);
        xyzz_add(acc, t);
    }
    for (int d = 16; d >= 1; d >>= 1) {
        xyzz_shfl_down(t, acc, d);
        xyzz_add(acc, t);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) xyzz_store(sm[warp], acc);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int k = 1; k < nw; ++k) {
            xyzz_load(t, sm[k]);
            xyzz_add(acc, t);
        }
        xyzz_store(wins + (size_t)w * 4 * F::N, acc);
    }
}

// Horner over windows, then affine + wire (+ compressed for BLS12-381).
template <class C>
__global__ void k_combine(const uint32_t* __restrict__ wins, int W, int c,
                          uint8_t* __restrict__ out_wire, uint8_t* __restrict__ out_comp) {
    using F = typename C::F;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Xyzz<F> acc, t;
    xyzz_load(acc, wins + (size_t)(W - 1) * 4 * F::N);
    for (int w = W - 2; w >= 0; --w) {
        for (int k = 0; k < c; ++k) xyzz_dbl(acc, acc);
        xyzz_load(t, wins + (size_t)w * 4 * F::N);
        xyzz_add(acc, t);
    }
    Affine<F> a;
    const bool fin = xyzz_to_affine(a, acc);
    Fe<F> x, y;
    if (fin) {
        fe_from_mont(x, a.x);
        fe_from_mont(y, a.y);
        fe_to_be_bytes(out_wire, x);
        fe_to_be_bytes(out_wire + F::BYTES, y);
    } else {
        for (int i = 0; i < C::WIRE; ++i) out_wire[i] = 0;
    }
    if (out_comp && C::CURVE_ID == 2) {
        // ZCash/IETF compressed form: bit7 compressed, bit6 infinity,
        // bit5 iff y > (p-1)/2, i.e. 2y > p.
        if (!fin) {
            out_comp[0] = 0xC0;
            for (int i = 1; i < 48; ++i) out_comp[i] = 0;
        } else {
            uint32_t d[F::N];
            // 2y - p - 1 >= 0  <=>  2y > p ; 2y < 2^(32N) since p < 2^(32N-1)
            uint32_t y2[F::N];
            uint32_t carry = 0;
            for (int i = 0; i < F::N; ++i) {
                uint64_t v = ((uint64_t)y.v[i] << 1) | carry;
                y2[i] = (uint32_t)v;
                carry = y.v[i] >> 31;
            }
            int64_t bw = 0;
            for (int i = 0; i < F::N; ++i) {
                int64_t v = (int64_t)y2[i] - (int64_t)F::P(i) - bw;
                d[i] = (uint32_t)v;
                bw = v < 0 ? 1 : 0;
            }
            bool nonzero = false;
            for (int i = 0; i < F::N; ++i) nonzero |= d[i] != 0;
            const bool larger = (bw == 0) && nonzero;  // 2y > p
            for (int i = 0; i < 48; ++i) out_comp[i] = out_wire[i];
            out_comp[0] |= 0x80;
            if (larger) out_comp[0] |= 0x20;
        }
    }
}

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------

constexpr int N_STAGE_EVENTS = 7;

struct MsmEngine {
    int curve;
    cudaEvent_t ev[N_STAGE_EVENTS] = {};
    bool ev_ready = false;
    bool ev_recorded = false;
    void mark(int i, cudaStream_t st) {
        if (!profiling_enabled()) return;
        if (!ev_ready) {
            for (auto& e : ev) KB_CUDA(cudaEventCreate(&e));
            ev_ready = true;
        }
        KB_CUDA(cudaEventRecord(ev[i], st));
        if (i == N_STAGE_EVENTS - 1) ev_recorded = true;
    }
    DevBuf table, keys, vals, counts, offsets, cursor, sorted, segoff, bid, part0, part1, buckets,
        groups, wins, scan_tmp;
};

int table_words(int curve) { return curve == 2 ? 2 * FpBLS::N : 2 * FpBN::N; }

MsmEngine* msm_engine_create(int curve) {
    MsmEngine* e = new MsmEngine();
    e->curve = curve;
    return e;
}

void msm_engine_destroy(MsmEngine* e) {
    if (!e) return;
    if (e->ev_ready)
        for (auto& ev : e->ev) cudaEventDestroy(ev);
    for (DevBuf* b : {&e->table, &e->keys, &e->vals, &e->counts, &e->offsets, &e->cursor,
                      &e->sorted, &e->segoff, &e->bid, &e->part0, &e->part1, &e->buckets,
                      &e->groups, &e->wins, &e->scan_tmp})
        b->release();
    delete e;
}

size_t msm_scratch_bytes(int curve, size_t n) {
    MsmOptions opt;
    MsmPlan p = make_msm_plan(curve, n, opt);
    const size_t N = curve == 2 ? 12 : 8;
    const size_t L = n * (size_t)p.W;
    size_t bytes = n * 2 * N * 4;                 // table
    bytes += 3 * L * 4;                           // keys, vals, sorted
    bytes += 4 * ((size_t)p.B + 1) * 4;           // counts, offsets, cursor, segoff
    bytes += p.seg_cap * 4;                       // bid
    bytes += 2 * p.seg_cap * 4 * N * 4;           // partials
    bytes += (size_t)p.B * 4 * N * 4;             // buckets
    bytes += (size_t)p.W * p.G * 4 * N * 4;       // groups
    return bytes + (1u << 20);
}

template <class C>
static void run_impl(MsmEngine* e, const uint8_t* d_scalars, const uint32_t* d_table, size_t n,
                     uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t st,
                     const MsmOptions& opt) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;  // words per XYZZ point
    if (n == 0) {
        KB_CUDA(cudaMemsetAsync(d_out_wire, 0, C::WIRE, st));
        if (d_out_comp) {
            KB_CUDA(cudaMemsetAsync(d_out_comp, 0, 48, st));
            KB_CUDA(cudaMemsetAsync(d_out_comp, 0xC0, 1, st));
        }
        return;
    }
    const MsmPlan p = make_msm_plan(C::CURVE_ID, n, opt);
    const size_t L = n * (size_t)p.W;
    if (n >= (1ull << 31) || L >= 0xffffffffull)
        throw std::invalid_argument("msm: n too large for 32-bit entry indices");
    e->keys.reserve(L * 4, st);
    e->vals.reserve(L * 4, st);
    e->sorted.reserve(L * 4, st);
    e->counts.reserve(((size_t)p.B + 1) * 4, st);
    e->offsets.reserve(((size_t)p.B + 1) * 4, st);
    e->cursor.reserve(((size_t)p.B + 1) * 4, st);
    e->segoff.reserve(((size_t)p.B + 1) * 4, st);
    e->bid.reserve(p.seg_cap * 4, st);
    e->part0.reserve(p.seg_cap * PW * 4, st);
    if (p.levels > 1) e->part1.reserve(p.seg_cap * PW * 4, st);
    e->buckets.reserve((size_t)p.B * PW * 4, st);
    e->groups.reserve((size_t)p.W * p.G * PW * 4, st);
    e->wins.reserve((size_t)p.W * PW * 4, st);
    e->scan_tmp.reserve(scan_tmp_words((size_t)p.B + 1) * 4, st);

    const int TB = 256;
    const int quirk = opt.ref_carry_quirk ? reference_best_c(n) : 0;
    e->mark(1, st);
    k_recode<C><<<ceil_div_u(n, TB), TB, 0, st>>>(reinterpret_cast<const uint32_t*>(d_scalars),
                                                   d_table, n, p.c, p.W, p.M, quirk,
                                                   e->keys.as<uint32_t>(), e->vals.as<uint32_t>());
    KB_LAUNCH_CHECK();
    e->mark(2, st);
    KB_CUDA(cudaMemsetAsync(e->counts.ptr, 0, ((size_t)p.B + 1) * 4, st));
    k_histogram<<<ceil_div_u(L, TB), TB, 0, st>>>(e->keys.as<uint32_t>(), L, e->counts.as<uint32_t>());
    KB_LAUNCH_CHECK();
    exclusive_scan_u32(e->counts.as<uint32_t>(), e->offsets.as<uint32_t>(), p.B, 0,
                       e->scan_tmp.as<uint32_t>(), st);
    KB_CUDA(cudaMemcpyAsync(e->cursor.ptr, e->offsets.ptr, (size_t)p.B * 4,
                            cudaMemcpyDeviceToDevice, st));
    k_scatter<<<ceil_div_u(L, TB), TB, 0, st>>>(e->keys.as<uint32_t>(), e->vals.as<uint32_t>(), L,
                                                 e->cursor.as<uint32_t>(), e->sorted.as<uint32_t>());
    KB_LAUNCH_CHECK();
    exclusive_scan_u32(e->counts.as<uint32_t>(), e->segoff.as<uint32_t>(), p.B, (uint32_t)p.K,
                       e->scan_tmp.as<uint32_t>(), st);
    KB_CUDA(cudaMemsetAsync(e->buckets.ptr, 0, (size_t)p.B * PW * 4, st));
    e->mark(3, st);
    const int TA = 128;
    k_accumulate<C><<<ceil_div_u(p.seg_cap, TA), TA, 0, st>>>(
        e->sorted.as<uint32_t>(), e->offsets.as<uint32_t>(), e->segoff.as<uint32_t>(), p.B,
        d_table, p.K, p.seg_cap, e->part0.as<uint32_t>(), e->bid.as<uint32_t>(),
        e->buckets.as<uint32_t>());
    KB_LAUNCH_CHECK();
    e->mark(4, st);
    uint32_t* in = e->part0.as<uint32_t>();
    uint32_t* out = e->part1.as<uint32_t>();
    for (int l = 2; l <= p.levels + 1; ++l) {
        k_fold<C><<<ceil_div_u(p.seg_cap, TA), TA, 0, st>>>(
            l, e->bid.as<uint32_t>(), e->segoff.as<uint32_t>(), p.B, p.K2, p.seg_cap, in, out,
            e->buckets.as<uint32_t>());
        KB_LAUNCH_CHECK();
        std::swap(in, out);
    }
    e->mark(5, st);
    const size_t ng = (size_t)p.W * p.G;
    k_reduce_groups<C><<<ceil_div_u(ng, TA), TA, 0, st>>>(e->buckets.as<uint32_t>(), p.W, p.M,
                                                           p.S, p.G, e->groups.as<uint32_t>());
    KB_LAUNCH_CHECK();
    k_window_sums<C><<<p.W, 256, 0, st>>>(e->groups.as<uint32_t>(), p.G, e->wins.as<uint32_t>());
    KB_LAUNCH_CHECK();
    k_combine<C><<<1, 32, 0, st>>>(e->wins.as<uint32_t>(), p.W, p.c, d_out_wire, d_out_comp);
    KB_LAUNCH_CHECK();
    e->mark(6, st);
}

void points_wire_to_table(int curve, const uint8_t* d_wire, uint32_t* d_table, size_t n,
                          cudaStream_t st) {
    if (n == 0) return;
    const int TB = 128;
    if (curve == 2)
        k_wire_to_table<G1BLS><<<ceil_div_u(n, TB), TB, 0, st>>>(d_wire, d_table, n);
    else
        k_wire_to_table<G1BN><<<ceil_div_u(n, TB), TB, 0, st>>>(d_wire, d_table, n);
    KB_LAUNCH_CHECK();
}

void points_table_to_wire(int curve, const uint32_t* d_table, uint8_t* d_wire, size_t n,
                          cudaStream_t st) {
    if (n == 0) return;
    const int TB = 128;
    if (curve == 2)
        k_table_to_wire<G1BLS><<<ceil_div_u(n, TB), TB, 0, st>>>(d_table, d_wire, n);
    else
        k_table_to_wire<G1BN><<<ceil_div_u(n, TB), TB, 0, st>>>(d_table, d_wire, n);
    KB_LAUNCH_CHECK();
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

void msm_run_table(MsmEngine* e, const uint8_t* d_scalars, const uint32_t* d_table, size_t n,
                   uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t st,
                   const MsmOptions& opt) {
    if (e->curve == 2)
        run_impl<G1BLS>(e, d_scalars, d_table, n, d_out_wire, d_out_comp, st, opt);
    else
        run_impl<G1BN>(e, d_scalars, d_table, n, d_out_wire, d_out_comp, st, opt);
}

void msm_run_wire(MsmEngine* e, const uint8_t* d_scalars, const uint8_t* d_points, size_t n,
                  uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t st,
                  const MsmOptions& opt) {
    const int tw = table_words(e->curve);
    e->table.reserve((n ? n : 1) * (size_t)tw * 4, st);
    e->mark(0, st);
    points_wire_to_table(e->curve, d_points, e->table.as<uint32_t>(), n, st);
    msm_run_table(e, d_scalars, e->table.as<uint32_t>(), n, d_out_wire, d_out_comp, st, opt);
}

}  // namespace kb200
