// Fr NTT kernels and host driver.  See ntt.cuh for the contract and the
// pass structure.
#include "../../include/kinet_b200/crypto_b200.h"
#include "field.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

#include "msm_desc.cuh"

#include <map>
#include <mutex>
#include <vector>

namespace kb200 {

namespace {

constexpr int NTT_THREADS = 1024;  // launch bound; passes of radix <= 2^10 run 256-thread blocks
// Tile of a pass with radix R <= 2^10: 1024 elements (32 KiB) per 256-thread
// block, four blocks per SM, so one block's stage barriers overlap the
// others' products.  Measured against one 4096-element, 1024-thread block per
// SM: BLS12-381 2^24 forward + inverse 13.67 -> 11.52 ms, BN254 2^26 coset
// 62.4 -> 54.1 ms, 2^16 0.33 -> 0.12 ms.  Radix 2^11 and 2^12 (single-pass
// transforms, e.g. the 4096-point blob) keep 4096-element, 1024-thread blocks.
constexpr int NTT_SMALL_THREADS = 256;
constexpr int NTT_SMALL_LOG_TILE = 10;
constexpr int NTT_SMEM_ELTS = 4096;  // 128 KiB of 32-byte elements per block
constexpr int TAB_SPLIT = 13;        // two-level tables: e = hi * 2^13 + lo

template <class F>
struct FrInfo;
template <>
struct FrInfo<FrBLS> {
    static constexpr uint32_t GEN = 7;
    static constexpr int ADICITY = 32;
    static constexpr int REDUCE_STEPS = 2;  // 2^256 < 3r
};
template <>
struct FrInfo<FrBN> {
    static constexpr uint32_t GEN = 5;
    static constexpr int ADICITY = 28;
    static constexpr int REDUCE_STEPS = 5;  // 2^256 < 6r
};

using Elt = Fe<FrBLS>;  // layout only (8 words); arithmetic is per field

template <class F>
KB_DEV void ld_elt(Fe<F>& a, const uint32_t* p) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 u = q[0], v = q[1];
    a.v[0] = u.x; a.v[1] = u.y; a.v[2] = u.z; a.v[3] = u.w;
    a.v[4] = v.x; a.v[5] = v.y; a.v[6] = v.z; a.v[7] = v.w;
}
template <class F>
KB_DEV void st_elt(uint32_t* p, const Fe<F>& a) {
    uint4* q = reinterpret_cast<uint4*>(p);
    q[0] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
    q[1] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

// x mod r for any 256-bit x, by bounded conditional subtraction.
template <class F>
KB_DEV void fr_reduce_full(Fe<F>& a) {
#pragma unroll
    for (int s = 0; s < FrInfo<F>::REDUCE_STEPS; ++s) reduce_once<F>(a, a.v);
}

template <class F>
KB_DEV void fe_pow_u64(Fe<F>& r, const Fe<F>& base, unsigned long long e) {
    Fe<F> acc, b = base;
    fe_one(acc);
    while (e) {
        if (e & 1) fe_mul(acc, acc, b);
        e >>= 1;
        if (e) fe_sqr(b, b);
    }
    r = acc;
}

// out = g^E (Montgomery form) for an 8-word exponent E; one thread.
template <class F>
__global__ void k_pow_gen(const uint32_t* __restrict__ exp, uint32_t* __restrict__ out) {
    if (threadIdx.x || blockIdx.x) return;
    Fe<F> g, acc;
    fe_zero(g);
    g.v[0] = FrInfo<F>::GEN;
    fe_to_mont(g, g);
    fe_one(acc);
    for (int w = 7; w >= 0; --w)
        for (int b = 31; b >= 0; --b) {
            fe_sqr(acc, acc);
            if ((exp[w] >> b) & 1u) fe_mul(acc, acc, g);
        }
    st_elt(out, acc);
}

// out[e] = base^(e * mult) for e < count (Montgomery form).
template <class F>
__global__ void k_powers(const uint32_t* __restrict__ base, unsigned long long mult, size_t count,
                         uint32_t* __restrict__ out) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    Fe<F> b, r;
    ld_elt(b, base);
    fe_pow_u64(r, b, (unsigned long long)e * mult);
    st_elt(out + e * 8, r);
}

// tw[e] = hi[e >> 13] * lo[e & 8191].
template <class F>
__global__ void k_combine_tables(const uint32_t* __restrict__ hi, const uint32_t* __restrict__ lo,
                                 size_t count, uint32_t* __restrict__ out) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    Fe<F> a, b, r;
    ld_elt(a, hi + (e >> TAB_SPLIT) * 8);
    ld_elt(b, lo + (e & ((1u << TAB_SPLIT) - 1)) * 8);
    fe_mul(r, a, b);
    st_elt(out + e * 8, r);
}

// out[e] = in[e] * s for e < count; s given in standard form (converted here).
template <class F>
__global__ void k_scale_table(uint32_t* __restrict__ t, size_t count, const uint32_t* __restrict__ s_std) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    Fe<F> s, a;
    ld_elt(s, s_std);
    fe_to_mont(s, s);
    ld_elt(a, t + e * 8);
    fe_mul(a, a, s);
    st_elt(t + e * 8, a);
}

struct PassArgs {
    const uint32_t* in;
    uint32_t* out;
    const uint32_t* tw;   // w_NT^e, e < NT (Montgomery form)
    int log_nt;
    int log_n;
    int log_R;            // radix of this pass
    int log_m;            // m_p = stride of the columns
    int log_mprev;        // m_{p-1} = block size
    int log_cb;           // columns (or rows) per CUDA block
    int inverse;
    int first;            // first pass: reduce inputs, optional coset pre-scale
    int final;            // last pass: digit-reversed store with post-scale
    int log_R1;           // R_1 (final pass index mapping)
    int nrest;            // final pass: number of "rest" digit values
    // coset / scale tables (Montgomery form), two-level split at 2^13
    const uint32_t* pre_hi;
    const uint32_t* pre_lo;
    const uint32_t* post_hi;
    const uint32_t* post_lo;
    const uint32_t* post_const;  // inverse without coset: n^-1
    size_t batch_stride;         // elements between consecutive vectors
    const unsigned long long* vec_off;  // if set: element offset of vector y
};

template <class F>
KB_DEV void two_level(Fe<F>& r, const uint32_t* hi, const uint32_t* lo, size_t e) {
    Fe<F> a, b;
    ld_elt(a, hi + (e >> TAB_SPLIT) * 8);
    ld_elt(b, lo + (e & ((1u << TAB_SPLIT) - 1)) * 8);
    fe_mul(r, a, b);
}

template <class F>
KB_DEV void twiddle(Fe<F>& w, const uint32_t* tw, int log_nt, size_t e_nt, int inverse) {
    const size_t NT = (size_t)1 << log_nt;
    size_t idx = e_nt & (NT - 1);
    if (inverse && idx) idx = NT - idx;
    ld_elt(w, tw + idx * 8);
}

__device__ __forceinline__ unsigned bitrev(unsigned x, int bits) {
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

// One pass.  Grid: x = CUDA blocks within one vector, y = vector in batch.
template <class F>
__global__ void __launch_bounds__(NTT_THREADS) k_ntt_pass(PassArgs a) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* sm = smem;                                  // cb * R elements
    uint32_t* stw = smem + ((size_t)8 << (a.log_cb + a.log_R));  // R/2 twiddles
    const int R = 1 << a.log_R, cb = 1 << a.log_cb;
    const size_t vec = a.vec_off ? (size_t)a.vec_off[blockIdx.y]
                                 : (size_t)blockIdx.y * a.batch_stride;
    const uint32_t* in = a.in + vec * 8;
    uint32_t* out = a.out + vec * 8;
    const int tot = R * cb;

    // Shared twiddles w_R^x (x < R/2): index x * NT / R in the big table.
    for (int x = threadIdx.x; x < R / 2; x += blockDim.x) {
        Fe<F> w;
        twiddle(w, a.tw, a.log_nt, (size_t)x << (a.log_nt - a.log_R), a.inverse);
        st_elt(stw + x * 8, w);
    }

    // Which columns / rows does this CUDA block own?
    size_t q = 0, col0 = 0, rest = 0, j1base = 0;
    if (!a.final) {
        const size_t ncolblk = ((size_t)1 << a.log_m) >> a.log_cb;
        q = blockIdx.x / ncolblk;
        col0 = (blockIdx.x % ncolblk) << a.log_cb;
    } else {
        const size_t nj1blk = ((size_t)1 << a.log_R1) >> a.log_cb;
        rest = blockIdx.x / nj1blk;
        j1base = (blockIdx.x % nj1blk) << a.log_cb;
    }

    // Load.
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        size_t g;
        int slot;
        if (!a.final) {
            const int c = e & (cb - 1), ih = e >> a.log_cb;
            g = (q << a.log_mprev) + ((size_t)ih << a.log_m) + col0 + c;
            slot = (c << a.log_R) + ih;
        } else {
            const int r = e >> a.log_R, ih = e & (R - 1);
            // rows of the final pass: q_r = j1 * (m_1 / R_P) + rest
            const size_t j1 = j1base + r;
            const int log_rows_per_j1 = a.log_n - a.log_R1 - a.log_R;
            g = (((j1 << log_rows_per_j1) + rest) << a.log_R) + ih;
            slot = e;
        }
        Fe<F> x;
        ld_elt(x, in + g * 8);
        if (a.first) {
            fr_reduce_full(x);
            if (a.pre_hi) {
                Fe<F> s;
                two_level(s, a.pre_hi, a.pre_lo, g);
                fe_mul(x, x, s);
            }
        }
        st_elt(sm + (size_t)slot * 8, x);
    }
    __syncthreads();

    // Radix-2 DIF stages on each of the cb sub-vectors of length R.  When
    // every thread has the same number `per` of butterflies per stage, warp w
    // takes butterflies [32 per w, 32 per (w + 1)), so from half-length
    // 32 per down a warp's butterflies touch only its own 64 per consecutive
    // elements of one sub-vector (or whole sub-vectors when R / 2 <= 32 per),
    // at that stage and the next: the warp alone consumes what it wrote, and
    // only the warp synchronises.  Every other stage, and the last (the store
    // reads any element), synchronise the block.
    const int half_total = tot >> 1;
    const int per = (half_total >= (int)blockDim.x && half_total % (int)blockDim.x == 0)
                        ? half_total / (int)blockDim.x
                        : 0;
    const int log_local = 5 + (per > 1 ? 31 - __clz(per) : 0);
    auto butterfly = [&](int s, int log_half, int b) {
        const int c = b >> (a.log_R - 1);
        const int bb = b & ((R >> 1) - 1);
        const int j = bb & ((1 << log_half) - 1);
        const int i0 = ((bb >> log_half) << (log_half + 1)) + j;
        const int i1 = i0 + (1 << log_half);
        uint32_t* p0 = sm + (size_t)((c << a.log_R) + i0) * 8;
        uint32_t* p1 = sm + (size_t)((c << a.log_R) + i1) * 8;
        Fe<F> u, v, t;
        ld_elt(u, p0);
        ld_elt(v, p1);
        fe_add(t, u, v);
        fe_sub(v, u, v);
        if (j) {
            Fe<F> w;
            ld_elt(w, stw + (size_t)(j << s) * 8);
            fe_mul(v, v, w);
        }
        st_elt(p0, t);
        st_elt(p1, v);
    };
    for (int s = 0; s < a.log_R; ++s) {
        const int log_half = a.log_R - 1 - s;
        if (per) {
            const int b0 = (int)(threadIdx.x >> 5) * per * 32 + (int)(threadIdx.x & 31);
            for (int k = 0; k < per; ++k) butterfly(s, log_half, b0 + 32 * k);
        } else {
            for (int b = threadIdx.x; b < half_total; b += blockDim.x) butterfly(s, log_half, b);
        }
        if (log_half <= (per ? log_local : 5) && s + 1 < a.log_R)
            __syncwarp();
        else
            __syncthreads();
    }

    // Store: DFT output j of sub-vector c sits at bitrev(j).
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        Fe<F> x;
        if (!a.final) {
            const int c = e & (cb - 1), j = e >> a.log_cb;
            ld_elt(x, sm + (size_t)((c << a.log_R) + (int)bitrev(j, a.log_R)) * 8);
            const size_t ilo = col0 + c;
            if (ilo && j) {
                // w_{m_{p-1}}^(ilo * j) = w_NT^(ilo * j * NT / m_{p-1})
                Fe<F> w;
                twiddle(w, a.tw, a.log_nt, (ilo * (size_t)j) << (a.log_nt - a.log_mprev), a.inverse);
                fe_mul(x, x, w);
            }
            const size_t g = (q << a.log_mprev) + ((size_t)j << a.log_m) + ilo;
            st_elt(out + g * 8, x);
        } else {
            const int r = e & (cb - 1), j = e >> a.log_cb;
            ld_elt(x, sm + (size_t)((r << a.log_R) + (int)bitrev(j, a.log_R)) * 8);
            const size_t j1 = j1base + r;
            const size_t X = j1 + (rest << a.log_R1) + ((size_t)j << (a.log_n - a.log_R));
            if (a.post_hi) {
                Fe<F> s;
                two_level(s, a.post_hi, a.post_lo, X);
                fe_mul(x, x, s);
            } else if (a.post_const) {
                Fe<F> s;
                ld_elt(s, a.post_const);
                fe_mul(x, x, s);
            }
            st_elt(out + X * 8, x);
        }
    }
}

}  // namespace

struct NttEngine {
    int curve;
    int log_nt = -1;             // twiddle table covers sizes up to 2^log_nt
    DevBuf tw, tw_hi, tw_lo, scratch, consts, ninv, pre_hi, pre_lo, post_hi;
    std::map<int, DevBuf> post_lo;  // per log n: n^-1 * g^-e, e < 2^13
    bool consts_ready = false;
    bool coset_ready = false;
    ~NttEngine() {
        for (DevBuf* b : {&tw, &tw_hi, &tw_lo, &scratch, &consts, &ninv, &pre_hi, &pre_lo, &post_hi})
            b->release();
        for (auto& kv : post_lo) kv.second.release();
    }
};

int ntt_max_log(int curve) { return curve == 2 ? 28 : 28; }

static std::mutex g_ntt_tune_mu;
static int g_ntt_tune[3][32];

void ntt_tune_set(int curve, int log_n, int log_r1) {
    if (curve < 1 || curve > 2 || log_n < 0 || log_n >= 32) return;
    std::lock_guard<std::mutex> lk(g_ntt_tune_mu);
    g_ntt_tune[curve][log_n] = log_r1;
}

int ntt_tune_get(int curve, int log_n) {
    if (curve < 1 || curve > 2 || log_n < 0 || log_n >= 32) return 0;
    std::lock_guard<std::mutex> lk(g_ntt_tune_mu);
    return g_ntt_tune[curve][log_n];
}

NttEngine* ntt_engine_create(int curve) {
    NttEngine* e = new NttEngine();
    e->curve = curve;
    return e;
}

void ntt_engine_destroy(NttEngine* e) { delete e; }

namespace {

// (r - 1) >> k, or r - 2, as 8 little-endian words (host side).
template <class F>
void exp_words(uint32_t out[8], int mode, int k) {
    uint32_t r[8];
    for (int i = 0; i < 8; ++i) r[i] = F::P(i);
    if (mode == 0) {  // (r - 1) >> k
        r[0] -= 1;
        for (int s = 0; s < k; ++s)
            for (int i = 0; i < 8; ++i) r[i] = (r[i] >> 1) | (i + 1 < 8 ? (r[i + 1] << 31) : 0u);
    } else {          // r - 2, borrow propagated (BLS12-381 r ends in ...0001)
        uint32_t borrow = 2;
        for (int i = 0; i < 8; ++i) {
            const uint32_t v = r[i];
            r[i] = v - borrow;
            borrow = v < borrow ? 1u : 0u;
        }
    }
    for (int i = 0; i < 8; ++i) out[i] = r[i];
}

// n^-1 mod r = r - (r - 1) / n for n = 2^k, standard form.
template <class F>
void ninv_words(uint32_t out[8], int k) {
    uint32_t q[8], r[8];
    exp_words<F>(q, 0, k);
    for (int i = 0; i < 8; ++i) r[i] = F::P(i);
    uint64_t bw = 0;
    for (int i = 0; i < 8; ++i) {
        const uint64_t v = (uint64_t)r[i] - q[i] - bw;
        out[i] = (uint32_t)v;
        bw = (v >> 63) & 1;
    }
}

// out[i] = to_mont(in[i]) for i < count (standard -> Montgomery form).
template <class F>
__global__ void k_to_mont(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Fe<F> a;
    ld_elt(a, in + (size_t)i * 8);
    fe_to_mont(a, a);
    st_elt(out + (size_t)i * 8, a);
}

// consts slots (8 words each): 0 = w_NT, 1 = exponent scratch, 2 = g,
// 3 = g^-1, 4 = exponent scratch.  ninv[k] = Montgomery(2^-k), k <= 28.
// All set-up work synchronises the stream; once a size (and coset use) has
// been prepared, ntt_run queues kernels only, so it can be graph-captured.
template <class F>
void prepare_impl(NttEngine* e, int log_n, int coset, cudaStream_t st) {
    if (log_n > FrInfo<F>::ADICITY || log_n > ntt_max_log(e->curve))
        throw std::invalid_argument("ntt: size exceeds the field's 2-adicity");
    const int TB = 256;
    const int maxlog = ntt_max_log(e->curve);
    if (!e->consts_ready) {
        e->consts.reserve(8 * 8 * 4, st);
        e->ninv.reserve((size_t)(maxlog + 1) * 32 * 2, st);
        uint32_t* C = e->consts.as<uint32_t>();
        std::vector<uint32_t> nv((size_t)(maxlog + 1) * 8);
        for (int k = 0; k <= maxlog; ++k) ninv_words<F>(&nv[(size_t)k * 8], k);
        uint32_t* stage = e->ninv.as<uint32_t>() + (size_t)(maxlog + 1) * 8;
        KB_CUDA(cudaMemcpyAsync(stage, nv.data(), nv.size() * 4, cudaMemcpyHostToDevice, st));
        k_to_mont<F><<<1, 32, 0, st>>>(stage, e->ninv.as<uint32_t>(), maxlog + 1);
        KB_LAUNCH_CHECK();
        uint32_t one[8] = {1, 0, 0, 0, 0, 0, 0, 0}, ex[8];
        KB_CUDA(cudaMemcpyAsync(C + 8, one, 32, cudaMemcpyHostToDevice, st));
        k_pow_gen<F><<<1, 32, 0, st>>>(C + 8, C + 16);
        KB_LAUNCH_CHECK();
        exp_words<F>(ex, 1, 0);
        KB_CUDA(cudaMemcpyAsync(C + 32, ex, 32, cudaMemcpyHostToDevice, st));
        k_pow_gen<F><<<1, 32, 0, st>>>(C + 32, C + 24);
        KB_LAUNCH_CHECK();
        KB_CUDA(cudaStreamSynchronize(st));
        e->consts_ready = true;
    }
    uint32_t* C = e->consts.as<uint32_t>();
    const int need = log_n < 1 ? 1 : log_n;
    if (need > e->log_nt) {
        const int L = need;
        uint32_t ex[8];
        exp_words<F>(ex, 0, L);
        KB_CUDA(cudaMemcpyAsync(C + 8, ex, 32, cudaMemcpyHostToDevice, st));
        k_pow_gen<F><<<1, 32, 0, st>>>(C + 8, C + 0);
        KB_LAUNCH_CHECK();
        const size_t NT = (size_t)1 << L;
        const size_t nlo = (size_t)1 << TAB_SPLIT;
        const size_t nhi = (NT + nlo - 1) / nlo;
        e->tw_lo.reserve(nlo * 32, st);
        e->tw_hi.reserve(nhi * 32, st);
        e->tw.reserve(NT * 32, st);
        k_powers<F><<<ceil_div_u(nlo, TB), TB, 0, st>>>(C + 0, 1, nlo, e->tw_lo.as<uint32_t>());
        KB_LAUNCH_CHECK();
        k_powers<F><<<ceil_div_u(nhi, TB), TB, 0, st>>>(C + 0, nlo, nhi, e->tw_hi.as<uint32_t>());
        KB_LAUNCH_CHECK();
        k_combine_tables<F><<<ceil_div_u(NT, TB), TB, 0, st>>>(e->tw_hi.as<uint32_t>(),
                                                               e->tw_lo.as<uint32_t>(), NT,
                                                               e->tw.as<uint32_t>());
        KB_LAUNCH_CHECK();
        e->log_nt = L;
        KB_CUDA(cudaStreamSynchronize(st));
    }
    if (coset && !e->coset_ready) {
        const size_t nlo = (size_t)1 << TAB_SPLIT;
        const size_t nhi = (size_t)1 << (28 - TAB_SPLIT);
        e->pre_lo.reserve(nlo * 32, st);
        e->pre_hi.reserve(nhi * 32, st);
        e->post_hi.reserve(nhi * 32, st);
        k_powers<F><<<ceil_div_u(nlo, TB), TB, 0, st>>>(C + 16, 1, nlo, e->pre_lo.as<uint32_t>());
        KB_LAUNCH_CHECK();
        k_powers<F><<<ceil_div_u(nhi, TB), TB, 0, st>>>(C + 16, nlo, nhi, e->pre_hi.as<uint32_t>());
        KB_LAUNCH_CHECK();
        k_powers<F><<<ceil_div_u(nhi, TB), TB, 0, st>>>(C + 24, nlo, nhi, e->post_hi.as<uint32_t>());
        KB_LAUNCH_CHECK();
        e->coset_ready = true;
        KB_CUDA(cudaStreamSynchronize(st));
    }
    if (coset && !e->post_lo.count(log_n)) {
        // post_lo[e] = n^-1 * g^-e
        const size_t nlo = (size_t)1 << TAB_SPLIT;
        DevBuf& b = e->post_lo[log_n];
        b.reserve(nlo * 32, st);
        k_powers<F><<<ceil_div_u(nlo, TB), TB, 0, st>>>(C + 24, 1, nlo, b.as<uint32_t>());
        KB_LAUNCH_CHECK();
        uint32_t* stage = e->ninv.as<uint32_t>() + (size_t)(maxlog + 1) * 8 + (size_t)log_n * 8;
        k_scale_table<F><<<ceil_div_u(nlo, TB), TB, 0, st>>>(b.as<uint32_t>(), nlo, stage);
        KB_LAUNCH_CHECK();
        KB_CUDA(cudaStreamSynchronize(st));
    }
}

template <class F>
void run_impl(NttEngine* e, uint32_t* d, size_t n, int inverse, int coset, size_t batch,
              const unsigned long long* d_vec_off, uint32_t* d_scratch, cudaStream_t st) {
    if (n == 0 || batch == 0) return;
    if (n & (n - 1)) throw std::invalid_argument("ntt: n must be a power of two");
    int log_n = 0;
    while (((size_t)1 << log_n) < n) ++log_n;
    prepare_impl<F>(e, log_n, coset, st);

    // Radix split: P = 1 up to 2^12, 2 up to 2^20, else 3 (each <= 2^10);
    // the first-pass radix may come from the autotuner.
    int logs[3], P;
    const int tuned = ntt_tune_get(e->curve, log_n);
    if (log_n <= 12) {
        P = 1;
        logs[0] = log_n;
    } else if (log_n <= 20) {
        P = 2;
        logs[0] = (log_n + 1) / 2;
        if (tuned >= log_n - 10 && tuned <= 10 && tuned >= 1) logs[0] = tuned;
        logs[1] = log_n - logs[0];
    } else {
        P = 3;
        logs[0] = (log_n + 2) / 3;
        if (tuned >= log_n - 20 && tuned <= 10 && tuned >= 1) logs[0] = tuned;
        logs[1] = (log_n - logs[0] + 1) / 2;
        logs[2] = log_n - logs[0] - logs[1];
    }
    uint32_t* scr = d_scratch;
    if (P > 1 && !scr) {
        if (d_vec_off) throw std::invalid_argument("ntt: listed vectors need caller scratch");
        e->scratch.reserve(n * batch * 32, st);
        scr = e->scratch.as<uint32_t>();
    }
    // P == 1: in place on d (each CUDA block owns whole vectors).  P >= 2: the
    // first pass moves d -> scratch, middle passes run in place on scratch,
    // and the last pass writes the natural-order result back into d.  With a
    // vector list the scratch mirrors d's layout (same offsets).
    int log_mprev = log_n;
    for (int p = 0; p < P; ++p) {
        PassArgs a{};
        a.tw = e->tw.as<uint32_t>();
        a.log_nt = e->log_nt;
        a.log_n = log_n;
        a.log_R = logs[p];
        a.log_m = log_mprev - logs[p];
        a.log_mprev = log_mprev;
        a.inverse = inverse;
        a.first = (p == 0);
        a.final = (p == P - 1);
        a.log_R1 = (P == 1) ? 0 : logs[0];
        a.batch_stride = n;
        a.vec_off = d_vec_off;
        if (a.first && coset && !inverse) {
            a.pre_hi = e->pre_hi.as<uint32_t>();
            a.pre_lo = e->pre_lo.as<uint32_t>();
        }
        if (a.final && inverse) {
            if (coset) {
                a.post_hi = e->post_hi.as<uint32_t>();
                a.post_lo = e->post_lo[log_n].as<uint32_t>();
            } else {
                a.post_const = e->ninv.as<uint32_t>() + (size_t)log_n * 8;
            }
        }
        const bool small_tile = a.log_R <= NTT_SMALL_LOG_TILE;
        int log_cb = (small_tile ? NTT_SMALL_LOG_TILE : 12) - a.log_R;
        if (!a.final) {
            if (log_cb > a.log_m) log_cb = a.log_m;
        } else {
            if (log_cb > a.log_R1) log_cb = a.log_R1;
        }
        a.log_cb = log_cb;
        a.in = (P == 1 || p == 0) ? d : scr;
        a.out = (P == 1 || a.final) ? d : scr;
        const size_t nblk = ((size_t)1 << (log_n - a.log_R)) >> log_cb;
        const size_t smem = (((size_t)8 << (log_cb + a.log_R)) + ((size_t)8 << a.log_R) / 2) * 4 + 64;
        // Largest pass: 4096 data elements plus 2048 shared twiddles (a
        // single-pass 2^12 transform) = 192 KiB + 64 B.
        set_smem_attr((const void*)k_ntt_pass<F>,
                      ((size_t)8 * NTT_SMEM_ELTS + 8 * 2048) * 4 + 64);
        dim3 grid((unsigned)nblk, (unsigned)batch);
        k_ntt_pass<F><<<grid, small_tile ? NTT_SMALL_THREADS : NTT_THREADS, smem, st>>>(a);
        KB_LAUNCH_CHECK();
        log_mprev = a.log_m;
    }
}

}  // namespace

void ntt_prepare(NttEngine* e, size_t n, int coset, cudaStream_t st) {
    int log_n = 0;
    while (((size_t)1 << log_n) < n) ++log_n;
    if (e->curve == 2)
        prepare_impl<FrBLS>(e, log_n, coset, st);
    else
        prepare_impl<FrBN>(e, log_n, coset, st);
}

void ntt_run(NttEngine* e, uint32_t* d, size_t n, int inverse, int coset, size_t batch,
             cudaStream_t st) {
    if (e->curve == 2)
        run_impl<FrBLS>(e, d, n, inverse, coset, batch, nullptr, nullptr, st);
    else
        run_impl<FrBN>(e, d, n, inverse, coset, batch, nullptr, nullptr, st);
}

void ntt_run_list(NttEngine* e, uint32_t* d, size_t n, int inverse, int coset, size_t count,
                  const unsigned long long* d_vec_off, uint32_t* d_scratch, cudaStream_t st) {
    if (e->curve == 2)
        run_impl<FrBLS>(e, d, n, inverse, coset, count, d_vec_off, d_scratch, st);
    else
        run_impl<FrBN>(e, d, n, inverse, coset, count, d_vec_off, d_scratch, st);
}


// ---------------------------------------------------------------------------
// Allocation-free Fr NTT.
//
// Some callers cannot allocate device memory: a process whose device memory
// is reserved up front by another allocator (a framework's caching pool, a
// fixed arena), where cudaMalloc fails or fragments that reservation, and a
// latency-bound service that cannot afford the device-wide waits of
// cudaMalloc and cudaFree while other work runs.  For them
// ntt_fr_transform_noalloc keeps all its scratch --
// the transform buffer, the pass ping-pong buffer, the twiddle table, the
// coset tables and the constants -- in one file-scope device array of fixed
// size, so a call allocates nothing.  The limit is n <= 2^16 elements
// (6.8 MB of scratch); every GPU that loads this library holds the array
// until the process exits.
// ---------------------------------------------------------------------------

constexpr int NOALLOC_MAX_LOG = 16;
constexpr size_t NOALLOC_MAX_N = (size_t)1 << NOALLOC_MAX_LOG;
constexpr size_t NOALLOC_TAB = (size_t)1 << TAB_SPLIT;                    // 8192
constexpr size_t NOALLOC_HI = NOALLOC_MAX_N >> TAB_SPLIT;                  // 8
// Element (32-byte) offsets of the regions inside the array.
constexpr size_t NA_DATA = 0;
constexpr size_t NA_SCR = NA_DATA + NOALLOC_MAX_N;
constexpr size_t NA_TW = NA_SCR + NOALLOC_MAX_N;
constexpr size_t NA_PRE_LO = NA_TW + NOALLOC_MAX_N;
constexpr size_t NA_POST_LO = NA_PRE_LO + NOALLOC_TAB;
constexpr size_t NA_PRE_HI = NA_POST_LO + NOALLOC_TAB;
constexpr size_t NA_POST_HI = NA_PRE_HI + NOALLOC_HI;
constexpr size_t NA_CONST = NA_POST_HI + NOALLOC_HI;  // 8 constant slots
constexpr size_t NA_ELTS = NA_CONST + 8;

static __device__ __align__(256) uint32_t g_ntt_noalloc_scratch[NA_ELTS * 8];

namespace {

// Device address of the scratch array, resolved once per device (with that
// device current) by cudaGetSymbolAddress; host code must never use the
// array's name itself as a device address.
std::mutex g_na_mu;
std::map<int, uint32_t*> g_na_ptr;

uint32_t* noalloc_scratch() {
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_na_mu);
    auto it = g_na_ptr.find(dev);
    if (it != g_na_ptr.end()) return it->second;
    void* p = nullptr;
    KB_CUDA(cudaGetSymbolAddress(&p, g_ntt_noalloc_scratch));
    g_na_ptr[dev] = static_cast<uint32_t*>(p);
    return static_cast<uint32_t*>(p);
}

template <class F>
void noalloc_impl(uint8_t* h_data, size_t n, int inverse, int coset) {
    int log_n = 0;
    while (((size_t)1 << log_n) < n) ++log_n;
    uint32_t* base = noalloc_scratch();
    auto at = [&](size_t elt) { return base + elt * 8; };
    uint32_t* C = at(NA_CONST);  // slots: 0 w_n, 1 exponent, 2 g, 3 g^-1, 4 n^-1 std, 5 n^-1
    const cudaStream_t st = 0;   // legacy default stream; cudaMemcpy orders with it
    const int TB = 256;
    KB_CUDA(cudaMemcpy(at(NA_DATA), h_data, n * 32, cudaMemcpyHostToDevice));
    // Everything read below is written first in this call, so no region has
    // to start at zero and the previous call's contents never leak in.
    uint32_t ex[8];
    exp_words<F>(ex, 0, log_n);
    KB_CUDA(cudaMemcpy(C + 8, ex, 32, cudaMemcpyHostToDevice));
    k_pow_gen<F><<<1, 32, 0, st>>>(C + 8, C + 0);  // w_n
    KB_LAUNCH_CHECK();
    k_powers<F><<<ceil_div_u(n, TB), TB, 0, st>>>(C + 0, 1, n, at(NA_TW));
    KB_LAUNCH_CHECK();
    uint32_t ni[8];
    ninv_words<F>(ni, log_n);
    KB_CUDA(cudaMemcpy(C + 32, ni, 32, cudaMemcpyHostToDevice));
    k_to_mont<F><<<1, 32, 0, st>>>(C + 32, C + 40, 1);
    KB_LAUNCH_CHECK();
    if (coset) {
        uint32_t one[8] = {1, 0, 0, 0, 0, 0, 0, 0};
        KB_CUDA(cudaMemcpy(C + 8, one, 32, cudaMemcpyHostToDevice));
        k_pow_gen<F><<<1, 32, 0, st>>>(C + 8, C + 16);  // g
        KB_LAUNCH_CHECK();
        exp_words<F>(ex, 1, 0);
        KB_CUDA(cudaMemcpy(C + 8, ex, 32, cudaMemcpyHostToDevice));
        k_pow_gen<F><<<1, 32, 0, st>>>(C + 8, C + 24);  // g^-1
        KB_LAUNCH_CHECK();
        k_powers<F><<<ceil_div_u(NOALLOC_TAB, TB), TB, 0, st>>>(C + 16, 1, NOALLOC_TAB, at(NA_PRE_LO));
        KB_LAUNCH_CHECK();
        k_powers<F><<<1, 32, 0, st>>>(C + 16, NOALLOC_TAB, NOALLOC_HI, at(NA_PRE_HI));
        KB_LAUNCH_CHECK();
        k_powers<F><<<ceil_div_u(NOALLOC_TAB, TB), TB, 0, st>>>(C + 24, 1, NOALLOC_TAB, at(NA_POST_LO));
        KB_LAUNCH_CHECK();
        k_scale_table<F><<<ceil_div_u(NOALLOC_TAB, TB), TB, 0, st>>>(at(NA_POST_LO), NOALLOC_TAB, C + 32);
        KB_LAUNCH_CHECK();
        k_powers<F><<<1, 32, 0, st>>>(C + 24, NOALLOC_TAB, NOALLOC_HI, at(NA_POST_HI));
        KB_LAUNCH_CHECK();
    }
    // The same passes as the resident path, over the static buffers.
    int logs[2], P;
    if (log_n <= 12) {
        P = 1;
        logs[0] = log_n;
    } else {
        P = 2;
        logs[0] = (log_n + 1) / 2;
        logs[1] = log_n - logs[0];
    }
    uint32_t* d = at(NA_DATA);
    uint32_t* scr = at(NA_SCR);
    int log_mprev = log_n;
    for (int p = 0; p < P; ++p) {
        PassArgs a{};
        a.tw = at(NA_TW);
        a.log_nt = log_n;
        a.log_n = log_n;
        a.log_R = logs[p];
        a.log_m = log_mprev - logs[p];
        a.log_mprev = log_mprev;
        a.inverse = inverse;
        a.first = (p == 0);
        a.final = (p == P - 1);
        a.log_R1 = (P == 1) ? 0 : logs[0];
        a.batch_stride = n;
        if (a.first && coset && !inverse) {
            a.pre_hi = at(NA_PRE_HI);
            a.pre_lo = at(NA_PRE_LO);
        }
        if (a.final && inverse) {
            if (coset) {
                a.post_hi = at(NA_POST_HI);
                a.post_lo = at(NA_POST_LO);
            } else {
                a.post_const = C + 40;
            }
        }
        const bool small_tile = a.log_R <= NTT_SMALL_LOG_TILE;
        int log_cb = (small_tile ? NTT_SMALL_LOG_TILE : 12) - a.log_R;
        if (!a.final) {
            if (log_cb > a.log_m) log_cb = a.log_m;
        } else {
            if (log_cb > a.log_R1) log_cb = a.log_R1;
        }
        a.log_cb = log_cb;
        a.in = (P == 1 || p == 0) ? d : scr;
        a.out = (P == 1 || a.final) ? d : scr;
        const size_t nblk = ((size_t)1 << (log_n - a.log_R)) >> log_cb;
        const size_t smem = (((size_t)8 << (log_cb + a.log_R)) + ((size_t)8 << a.log_R) / 2) * 4 + 64;
        set_smem_attr((const void*)k_ntt_pass<F>, ((size_t)8 * NTT_SMEM_ELTS + 8 * 2048) * 4 + 64);
        k_ntt_pass<F><<<dim3((unsigned)nblk, 1), small_tile ? NTT_SMALL_THREADS : NTT_THREADS, smem, st>>>(a);
        KB_LAUNCH_CHECK();
        log_mprev = a.log_m;
    }
    KB_CUDA(cudaMemcpy(h_data, at(NA_DATA), n * 32, cudaMemcpyDeviceToHost));
}

}  // namespace

}  // namespace kb200

extern "C" int ntt_fr_transform_noalloc(int curve, uint8_t* coeffs32le, size_t n, int inverse,
                                        int coset) {
    using namespace kb200;
    if (!coeffs32le) return KB200_CRYPTO_ERR_INPUT;
    if (curve != 1 && curve != 2) return KB200_CRYPTO_ERR_INPUT;
    if (n == 0 || (n & (n - 1))) return KB200_CRYPTO_ERR_LENGTH;
    if (n > NOALLOC_MAX_N) {
        set_last_error("ntt_fr_transform_noalloc: n exceeds the 2^16-element static scratch "
                       "(use ntt_fr_forward / ntt_fr_inverse for larger transforms)");
        return KB200_CRYPTO_ERR_LENGTH;
    }
    try {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            set_last_error("no usable CUDA device (kinet-b200 has no CPU fallback)");
            return KB200_CRYPTO_ERR_BACKEND;
        }
        if (curve == 2)
            noalloc_impl<FrBLS>(coeffs32le, n, inverse, coset);
        else
            noalloc_impl<FrBN>(coeffs32le, n, inverse, coset);
        return KB200_CRYPTO_OK;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return KB200_CRYPTO_ERR_BACKEND;
    }
}

namespace kb200 {
}  // namespace kb200
