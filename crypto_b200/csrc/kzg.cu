// Fixed-base G1 multiplication and Fr powers.  See kzg.cuh.
#include "curve.cuh"
#include "kzg.cuh"
#include "msm.cuh"

#include <map>
#include <mutex>
#include "runtime.cuh"

namespace kb200 {

namespace {

// Generators, big-endian affine wire encoding.
// BLS12-381: bls/cpp/bls12_381_g1.hpp:205-218; BN254: (1, 2) (EIP-196).
__constant__ uint8_t GEN_BLS[96] = {
    0x17, 0xF1, 0xD3, 0xA7, 0x31, 0x97, 0xD7, 0x94, 0x26, 0x95, 0x63, 0x8C, 0x4F, 0xA9, 0xAC, 0x0F,
    0xC3, 0x68, 0x8C, 0x4F, 0x97, 0x74, 0xB9, 0x05, 0xA1, 0x4E, 0x3A, 0x3F, 0x17, 0x1B, 0xAC, 0x58,
    0x6C, 0x55, 0xE8, 0x3F, 0xF9, 0x7A, 0x1A, 0xEF, 0xFB, 0x3A, 0xF0, 0x0A, 0xDB, 0x22, 0xC6, 0xBB,
    0x08, 0xB3, 0xF4, 0x81, 0xE3, 0xAA, 0xA0, 0xF1, 0xA0, 0x9E, 0x30, 0xED, 0x74, 0x1D, 0x8A, 0xE4,
    0xFC, 0xF5, 0xE0, 0x95, 0xD5, 0xD0, 0x0A, 0xF6, 0x00, 0xDB, 0x18, 0xCB, 0x2C, 0x04, 0xB3, 0xED,
    0xD0, 0x3C, 0xC7, 0x44, 0xA2, 0x88, 0x8A, 0xE4, 0x0C, 0xAA, 0x23, 0x29, 0x46, 0xC5, 0xE7, 0xE1};
__constant__ uint8_t GEN_BN[64] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1,
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 2};

constexpr int FB_WINDOWS = 32;   // 8-bit windows over 256-bit scalars
constexpr int FB_ENTRIES = 255;  // d = 1..255

// bases[j] = 2^(8j) * G (XYZZ), one thread.
template <class C>
__global__ void k_fb_bases(uint32_t* __restrict__ bases) {
    using F = typename C::F;
    if (threadIdx.x || blockIdx.x) return;
    uint32_t w[2 * F::N];
    wire_to_table<C>(w, C::CURVE_ID == 2 ? GEN_BLS : GEN_BN);
    Affine<F> g;
    aff_load(g, w);
    Xyzz<F> acc;
    xyzz_from_affine(acc, g);
    for (int j = 0; j < FB_WINDOWS; ++j) {
        xyzz_store(bases + (size_t)j * 4 * F::N, acc);
        for (int k = 0; k < 8; ++k) xyzz_dbl(acc, acc);
    }
}

// table[j][d-1] = d * bases[j], affine Montgomery (2N words).
template <class C>
__global__ void k_fb_entries(const uint32_t* __restrict__ bases, uint32_t* __restrict__ table) {
    using F = typename C::F;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= FB_WINDOWS * FB_ENTRIES) return;
    const int j = t / FB_ENTRIES, d = t % FB_ENTRIES + 1;
    Xyzz<F> b, acc;
    xyzz_load(b, bases + (size_t)j * 4 * F::N);
    xyzz_set_inf(acc);
    for (int bit = 7; bit >= 0; --bit) {
        xyzz_dbl(acc, acc);
        if ((d >> bit) & 1) xyzz_add(acc, b);
    }
    Affine<F> a;
    xyzz_to_affine(a, acc);  // d * 2^(8j) * G is never infinity (d < r)
    fe_store(table + (size_t)t * 2 * F::N, a.x);
    fe_store(table + (size_t)t * 2 * F::N + F::N, a.y);
}

template <class C>
__global__ void __launch_bounds__(128) k_fb_mul(const uint32_t* __restrict__ table,
                                                const uint8_t* __restrict__ scalars, size_t n,
                                                uint32_t* __restrict__ out_table,
                                                uint8_t* __restrict__ out_wire) {
    using F = typename C::F;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* s = scalars + i * 32;
    Xyzz<F> acc;
    xyzz_set_inf(acc);
    for (int j = 0; j < FB_WINDOWS; ++j) {
        const int d = s[j];
        if (!d) continue;
        Affine<F> a;
        aff_load(a, table + (size_t)(j * FB_ENTRIES + d - 1) * 2 * F::N);
        xyzz_add_affine(acc, a);
    }
    Affine<F> a;
    const bool fin = xyzz_to_affine(a, acc);
    if (out_table) {
        uint32_t* o = out_table + i * 2 * F::N;
        if (fin) {
            fe_store(o, a.x);
            fe_store(o + F::N, a.y);
        } else {
            for (int k = 0; k < 2 * F::N; ++k) o[k] = 0;
            o[F::N - 1] = INF_FLAG;
        }
    }
    if (out_wire) {
        uint8_t* o = out_wire + i * C::WIRE;
        if (fin) {
            Fe<F> x, y;
            fe_from_mont(x, a.x);
            fe_from_mont(y, a.y);
            fe_to_be_bytes(o, x);
            fe_to_be_bytes(o + F::BYTES, y);
        } else {
            for (int k = 0; k < C::WIRE; ++k) o[k] = 0;
        }
    }
}

template <class F>
__global__ void k_fr_powers(const uint8_t* __restrict__ tau, size_t n, uint8_t* __restrict__ out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fe<F> t, acc;
    const uint32_t* tw = reinterpret_cast<const uint32_t*>(tau);
    for (int k = 0; k < F::N; ++k) t.v[k] = tw[k];
    fe_to_mont(t, t);
    fe_one(acc);
    unsigned long long e = i;
    Fe<F> b = t;
    while (e) {
        if (e & 1) fe_mul(acc, acc, b);
        e >>= 1;
        if (e) fe_sqr(b, b);
    }
    fe_from_mont(acc, acc);
    uint32_t* o = reinterpret_cast<uint32_t*>(out + i * 32);
    for (int k = 0; k < F::N; ++k) o[k] = acc.v[k];
}

// Levels 1..W-1 of a shifted table: level w row i = [2^(c w)] (base row i).
// One thread per point: c doublings per level, then the affine conversion
// with one inversion per block per level (Montgomery's trick: inclusive
// prefix and suffix products of ZZ*ZZZ across the block's 128 points, so
// 1/d_t = 1/(d_0...d_127) * P_{t-1} * S_{t+1}).
constexpr int SHIFT_T = 128;

template <class F>
__device__ __forceinline__ void smw_load(Fe<F>& r, const uint32_t* sm, int t) {
#pragma unroll
    for (int k = 0; k < F::N; ++k) r.v[k] = sm[k * SHIFT_T + t];
}
template <class F>
__device__ __forceinline__ void smw_store(uint32_t* sm, int t, const Fe<F>& a) {
#pragma unroll
    for (int k = 0; k < F::N; ++k) sm[k * SHIFT_T + t] = a.v[k];
}

__global__ void __launch_bounds__(SHIFT_T) k_shift_levels(const uint32_t* __restrict__ base, size_t n,
                                                          int c, int W, uint32_t* __restrict__ out) {
    using F = FpBLS;
    __shared__ uint32_t s_pre[SHIFT_T * F::N];
    __shared__ uint32_t s_suf[SHIFT_T * F::N];
    __shared__ uint32_t s_inv[F::N];
    const int t = threadIdx.x;
    const size_t i = (size_t)blockIdx.x * SHIFT_T + t;
    const bool live = i < n;
    bool inf = true;
    Xyzz<F> p;
    xyzz_set_inf(p);
    if (live) {
        const uint32_t* src = base + i * 2 * F::N;
        for (int k = 0; k < 2 * F::N; ++k) out[i * 2 * F::N + k] = src[k];
        inf = aff_is_inf_words<F>(src);
        if (!inf) {
            Affine<F> a;
            aff_load(a, src);
            xyzz_from_affine(p, a);
        }
    }
    for (int w = 1; w < W; ++w) {
        if (!inf) {
            for (int k = 0; k < c; ++k) xyzz_dbl(p, p);
            inf = xyzz_is_inf(p);
        }
        Fe<F> d;
        if (inf)
            fe_one(d);
        else
            fe_mul(d, p.ZZ, p.ZZZ);
        smw_store(s_pre, t, d);
        smw_store(s_suf, t, d);
        __syncthreads();
        for (int k = 1; k < SHIFT_T; k <<= 1) {
            Fe<F> a, b, o;
            smw_load(a, s_pre, t);
            smw_load(b, s_suf, t);
            if (t >= k) {
                smw_load(o, s_pre, t - k);
                fe_mul(a, a, o);
            }
            if (t + k < SHIFT_T) {
                smw_load(o, s_suf, t + k);
                fe_mul(b, b, o);
            }
            __syncthreads();
            smw_store(s_pre, t, a);
            smw_store(s_suf, t, b);
            __syncthreads();
        }
        if (t == 0) {
            Fe<F> tot, inv;
            smw_load(tot, s_pre, SHIFT_T - 1);
            fe_inv(inv, tot);
            fe_store(s_inv, inv);
        }
        __syncthreads();
        Fe<F> r, o;
        fe_load(r, s_inv);
        if (t > 0) {
            smw_load(o, s_pre, t - 1);
            fe_mul(r, r, o);
        }
        if (t + 1 < SHIFT_T) {
            smw_load(o, s_suf, t + 1);
            fe_mul(r, r, o);
        }
        if (live) {
            uint32_t* dst = out + ((size_t)w * n + i) * 2 * F::N;
            if (inf) {
                for (int k = 0; k < 2 * F::N; ++k) dst[k] = 0;
                dst[F::N - 1] = INF_FLAG;
            } else {
                Fe<F> iz, x, y;
                fe_mul(iz, r, p.ZZZ);  // 1/ZZ
                fe_mul(x, p.X, iz);
                fe_mul(iz, r, p.ZZ);   // 1/ZZZ
                fe_mul(y, p.Y, iz);
                fe_store(dst, x);
                fe_store(dst + F::N, y);
            }
        }
        __syncthreads();  // the scans of the next level reuse the arrays
    }
}

}  // namespace

struct ShiftTables {
    const uint32_t* base = nullptr;
    size_t n = 0;
    uint64_t generation = 0;
    std::map<int, DevBuf> levels;
    std::mutex mu;
};

ShiftTables* shift_tables_create() { return new ShiftTables(); }

void shift_tables_destroy(ShiftTables* t) {
    if (!t) return;
    for (auto& kv : t->levels) kv.second.release();
    delete t;
}

void shift_tables_reset(ShiftTables* t, const uint32_t* d_base, size_t n) {
    std::lock_guard<std::mutex> lk(t->mu);
    for (auto& kv : t->levels) kv.second.release();  // cudaFree waits for the device
    t->levels.clear();
    t->base = d_base;
    t->n = n;
    ++t->generation;
}

uint64_t shift_tables_generation(const ShiftTables* t) { return t->generation; }
size_t shift_tables_stride(const ShiftTables* t) { return t->n; }

// Cap on one shifted table (HBM is 180 GB; a 2^20-point table at c = 20 is 1.3 GB).
constexpr size_t SHIFT_TABLE_MAX_BYTES = (size_t)8 << 30;

const uint32_t* shift_tables_get(ShiftTables* t, int c, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(t->mu);
    if (!t->base || t->n == 0 || c < 2) return nullptr;
    auto it = t->levels.find(c);
    if (it != t->levels.end()) return it->second.as<uint32_t>();
    const int W = msm_windows_for(c);
    const size_t bytes = (size_t)W * t->n * 2 * FpBLS::N * 4;
    if (bytes > SHIFT_TABLE_MAX_BYTES) return nullptr;
    DevBuf& b = t->levels[c];
    b.reserve(bytes, st);
    k_shift_levels<<<ceil_div_u(t->n, SHIFT_T), SHIFT_T, 0, st>>>(t->base, t->n, c, W, b.as<uint32_t>());
    KB_LAUNCH_CHECK();
    KB_CUDA(cudaStreamSynchronize(st));  // usable from any stream once returned
    return b.as<uint32_t>();
}

static std::mutex g_commit_tune_mu;
static int g_commit_tune[48];

void commit_tune_set(int log_n, int c) {
    if (log_n < 0 || log_n >= 48 || (c != 0 && c != 13 && c != 16 && c != 19)) return;
    std::lock_guard<std::mutex> lk(g_commit_tune_mu);
    g_commit_tune[log_n] = c;
}

int commit_tune_get(int log_n) {
    if (log_n < 0 || log_n >= 48) return 0;
    std::lock_guard<std::mutex> lk(g_commit_tune_mu);
    return g_commit_tune[log_n];
}

int shift_c_for(const size_t* sizes, size_t count) {
    // A single commit: the autotuner's choice for its size class, if any.
    if (count == 1 && sizes[0]) {
        int lg = 0;
        while (((size_t)1 << lg) < sizes[0]) ++lg;
        if (const int t = commit_tune_get(lg)) return t;
    }
    // Accumulation: one entry per window canonical scalars populate;
    // reduction: ~7 entry-equivalents per bucket of the single shared window
    // of each item.  Only three window sizes are offered, so a
    // resident setup carries at most three shifted tables.
    int best_c = 13;
    double best = 1e300;
    for (int c : {13, 16, 19}) {
        const double wl = (double)((255 + c - 1) / c);
        double cost = 0;
        for (size_t i = 0; i < count; ++i) cost += wl * (double)sizes[i] + RED_COST * (double)(1u << (c - 1));
        if (cost < best) {
            best = cost;
            best_c = c;
        }
    }
    return best_c;
}

struct FixedBase {
    int curve;
    DevBuf bases, table;
};

FixedBase* fixed_base_create(int curve, cudaStream_t st) {
    FixedBase* fb = new FixedBase();
    fb->curve = curve;
    const int N = curve == 2 ? FpBLS::N : FpBN::N;
    fb->bases.reserve((size_t)FB_WINDOWS * 4 * N * 4, st);
    fb->table.reserve((size_t)FB_WINDOWS * FB_ENTRIES * 2 * N * 4, st);
    const int tot = FB_WINDOWS * FB_ENTRIES;
    if (curve == 2) {
        k_fb_bases<G1BLS><<<1, 32, 0, st>>>(fb->bases.as<uint32_t>());
        k_fb_entries<G1BLS><<<ceil_div_u(tot, 128), 128, 0, st>>>(fb->bases.as<uint32_t>(),
                                                                  fb->table.as<uint32_t>());
    } else {
        k_fb_bases<G1BN><<<1, 32, 0, st>>>(fb->bases.as<uint32_t>());
        k_fb_entries<G1BN><<<ceil_div_u(tot, 128), 128, 0, st>>>(fb->bases.as<uint32_t>(),
                                                                 fb->table.as<uint32_t>());
    }
    KB_LAUNCH_CHECK();
    KB_CUDA(cudaStreamSynchronize(st));
    return fb;
}

void fixed_base_destroy(FixedBase* fb) {
    if (!fb) return;
    fb->bases.release();
    fb->table.release();
    delete fb;
}

void fixed_base_mul(FixedBase* fb, const uint8_t* d_scalars, size_t n, uint32_t* d_table_out,
                    uint8_t* d_wire_out, cudaStream_t st) {
    if (n == 0) return;
    if (fb->curve == 2)
        k_fb_mul<G1BLS><<<ceil_div_u(n, 128), 128, 0, st>>>(fb->table.as<uint32_t>(), d_scalars,
                                                            n, d_table_out, d_wire_out);
    else
        k_fb_mul<G1BN><<<ceil_div_u(n, 128), 128, 0, st>>>(fb->table.as<uint32_t>(), d_scalars, n,
                                                           d_table_out, d_wire_out);
    KB_LAUNCH_CHECK();
}

void fr_powers(int curve, const uint8_t* d_tau, size_t n, uint8_t* d_out, cudaStream_t st) {
    if (n == 0) return;
    if (curve == 2)
        k_fr_powers<FrBLS><<<ceil_div_u(n, 256), 256, 0, st>>>(d_tau, n, d_out);
    else
        k_fr_powers<FrBN><<<ceil_div_u(n, 256), 256, 0, st>>>(d_tau, n, d_out);
    KB_LAUNCH_CHECK();
}

}  // namespace kb200
