// Word-prime NTT on the GPU, behind the reference's ntt_forward /
// ntt_inverse (ntt/c-abi/c_ntt.cpp:81-179).
//
// The reference has three bodies, and each is reproduced operation for
// operation, so results agree for every input (reduced or not, any root):
//
//   CYC   n <= 2^16, modulus 998244353, pinned root: data in standard form,
//         twiddles in Montgomery form with R = 2^32, 64-bit wrapping products
//         (ntt/cpp/ntt.cpp:52-66, 100-172).
//   SMALL n <= 2^16, any other (modulus, root): both butterfly inputs reduced
//         mod q, 128-bit products, an addition without overflow check
//         (ntt/cpp/ntt.cpp:33-45, 176-219).
//   LARGE 2^16 < n <= 2^20: six-step: column sub-NTTs, diagonal twiddles,
//         row sub-NTTs; output left in the transposed layout; the upper
//         butterfly input reduced by the product only, an overflow-checked
//         addition (ntt/cpp/ntt_large.cpp:28-44, 95-122, 145-248).
//
// Every body is a radix-2 decimation-in-time transform after a bit-reversal
// permutation.  On the device each pass loads whole lines (sub-transforms, or
// the 2^11-element blocks and columns of a longer one) into shared memory,
// applies the bit reversal on the load, runs its radix-2 stages with the
// same butterfly pairs and twiddles as the reference, applies the fused
// post-multiply (diagonal twiddles or 1/n) and stores.  Twiddles w^e come
// from two small tables (w^e = lo[e mod 2^h] * hi[e >> h]).
//
// Products use Montgomery multiplication with R = 2^64 for odd q (the result
// equals the reference's (a*b) % q for every a < 2^64, b < q), the
// reference's own R = 2^32 formulas on the CYC path, and shift-and-add
// products for even q.
#include <algorithm>
#include <cstring>
#include <map>
#include <stdexcept>
#include <tuple>
#include <vector>

#include "runtime.cuh"
#include "wntt.cuh"

namespace kb200 {
namespace {

// Cyclone-FFT prime, its pinned 2^16-th root and the Montgomery (R = 2^32)
// constant -q^-1 mod 2^32 (ntt/cpp/ntt.hpp:43-64).
constexpr uint64_t CYC_Q = 998244353ull;
constexpr uint64_t CYC_ROOT = 629671588ull;
constexpr uint64_t CYC_QINV32 = 998244351ull;
constexpr uint32_t CYC_MAX_LOG = 16;
constexpr uint32_t LARGE_MAX_LOG = 20;

enum WMode : int { W_CYC = 0, W_SMALL = 1, W_LARGE = 2 };

constexpr int WNTT_THREADS = 256;
constexpr uint32_t WNTT_TILE = 4096;  // words per CTA (32 KiB)
constexpr uint32_t WNTT_MAX_LINE_LOG = 11;

struct WArith {
    uint64_t q;
    uint64_t qinv;  // -q^-1 mod 2^64 (odd q)
    int mode;
    int even;       // q even: standard-form twiddles, shift-and-add products
};

struct WPass {
    const uint64_t* in;
    uint64_t* out;
    uint32_t lines, log_L, lpc;
    uint64_t in_ls, in_ts, out_ls, out_ts;  // word address = line * ls + t * ts
    uint32_t line_rev_bits;                 // source line index bit-reversed over this many bits
    int bitrev;                             // slot t <- source element bitrev(t)
    int reduce_in;                          // x mod q on load
    uint32_t s_lo, s_hi;                    // radix-2 stages (1-based, inclusive)
    uint32_t gl, log_gt;                    // stage position of (line, t): line * gl + (t << log_gt)
    uint32_t log_n;                         // twiddle of stage s, index j: w^(j << (log_n - s))
    const uint64_t* tw_lo;
    const uint64_t* tw_hi;
    uint32_t h;
    int post;                               // 0 none, 1: * w^(line * t), 2: * scale
    uint64_t scale;
};

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, uint32_t bits) {
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

__device__ __forceinline__ uint64_t cyc_redc(uint64_t t) {
    const uint64_t m = ((t & 0xffffffffull) * CYC_QINV32) & 0xffffffffull;
    const uint64_t u = (t + m * CYC_Q) >> 32;
    return u >= CYC_Q ? u - CYC_Q : u;
}

// a * b * 2^-64 mod q, canonical, for any a < 2^64 and b < q (q odd).
__device__ __forceinline__ uint64_t mont64(uint64_t a, uint64_t b, uint64_t q, uint64_t qinv) {
    const uint64_t lo = a * b, hi = __umul64hi(a, b);
    const uint64_t m = lo * qinv;
    const uint64_t mh = __umul64hi(m, q);
    // lo + m*q = 0 mod 2^64: the low half carries exactly when lo != 0.
    const uint64_t s = hi + mh;
    uint64_t c = s < hi;
    const uint64_t s1 = s + (lo != 0 ? 1ull : 0ull);
    c += s1 < s;
    return (c || s1 >= q) ? s1 - q : s1;
}

__device__ __forceinline__ uint64_t add_ovf(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    if (s >= q || s < a) s -= q;
    return s;
}

// (a * b) mod q for a, b < q, any q >= 1 (used for even q only).
__device__ __noinline__ uint64_t mulmod_slow(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t r = 0;
    for (int i = 63; i >= 0; --i) {
        r = add_ovf(r, r, q);
        if ((b >> i) & 1ull) r = add_ovf(r, a, q);
    }
    return r;
}

// Data word times a twiddle in the path's representation, canonical result
// (on the CYC path: the reference's mont_mul, wrapping product included).
__device__ __forceinline__ uint64_t tw_mul(const WArith& A, uint64_t a, uint64_t w) {
    if (A.mode == W_CYC) return cyc_redc(a * w);
    if (A.even) return mulmod_slow(a % A.q, w, A.q);
    return mont64(a, w, A.q, A.qinv);
}

__device__ __forceinline__ uint64_t tw_pow(const WArith& A, const WPass& p, uint64_t e) {
    return tw_mul(A, p.tw_lo[e & ((1ull << p.h) - 1ull)], p.tw_hi[e >> p.h]);
}

__device__ __forceinline__ void butterfly(const WArith& A, uint64_t& x0, uint64_t& x1, uint64_t w) {
    const uint64_t q = A.q;
    const uint64_t u = x0;
    const uint64_t t = tw_mul(A, x1, w);
    uint64_t s = u + t;
    if (A.mode == W_LARGE) {
        if (s >= q || s < u) s -= q;
    } else if (s >= q) {
        s -= q;
    }
    x0 = s;
    x1 = u >= t ? u - t : u + q - t;
}

__global__ void __launch_bounds__(WNTT_THREADS) k_wntt_pass(WArith A, WPass p) {
    __shared__ uint64_t sm[WNTT_TILE];
    __shared__ uint64_t stw[1u << (WNTT_MAX_LINE_LOG - 1)];
    const uint32_t L = 1u << p.log_L;
    const uint32_t line0 = blockIdx.x * p.lpc;
    if (line0 >= p.lines) return;
    const uint32_t nl = min(p.lpc, p.lines - line0);
    const uint32_t cnt = nl * L;
    for (uint32_t idx = threadIdx.x; idx < cnt; idx += blockDim.x) {
        uint32_t c, t;
        if (p.in_ls == 1) {
            c = idx % nl;
            t = idx / nl;
        } else {
            c = idx / L;
            t = idx % L;
        }
        const uint32_t line = line0 + c;
        const uint64_t sl = p.line_rev_bits ? brev_bits(line, p.line_rev_bits) : line;
        const uint32_t st = p.bitrev ? brev_bits(t, p.log_L) : t;
        uint64_t v = p.in[sl * p.in_ls + (uint64_t)st * p.in_ts];
        if (p.reduce_in) v %= A.q;
        sm[c * L + t] = v;
    }
    const bool local_tw = p.gl == 0 && p.log_gt == 0;
    if (local_tw && p.s_lo <= p.s_hi)
        for (uint32_t k = threadIdx.x; k < L / 2; k += blockDim.x)
            stw[k] = tw_pow(A, p, (uint64_t)k << (p.log_n - p.log_L));
    __syncthreads();
    const uint32_t half_line = L / 2;
    for (uint32_t s = p.s_lo; s <= p.s_hi; ++s) {
        const uint32_t half = 1u << (s - 1 - p.log_gt);  // pair distance in t
        for (uint32_t b = threadIdx.x; b < cnt / 2; b += blockDim.x) {
            const uint32_t c = b / half_line, r = b % half_line;
            const uint32_t t0 = (r / half) * 2 * half + (r % half);
            const uint32_t i0 = c * L + t0;
            uint64_t w;
            if (local_tw) {
                w = stw[(r % half) << (p.log_L - s)];
            } else {
                const uint64_t g = (uint64_t)(line0 + c) * p.gl + ((uint64_t)t0 << p.log_gt);
                const uint64_t j = g & ((1ull << (s - 1)) - 1ull);
                w = tw_pow(A, p, j << (p.log_n - s));
            }
            butterfly(A, sm[i0], sm[i0 + half], w);
        }
        __syncthreads();
    }
    for (uint32_t idx = threadIdx.x; idx < cnt; idx += blockDim.x) {
        uint32_t c, t;
        if (p.out_ls == 1) {
            c = idx % nl;
            t = idx / nl;
        } else {
            c = idx / L;
            t = idx % L;
        }
        const uint32_t line = line0 + c;
        uint64_t v = sm[c * L + t];
        if (p.post == 1)
            v = tw_mul(A, v, tw_pow(A, p, (uint64_t)line * t));
        else if (p.post == 2)
            v = tw_mul(A, v, p.scale);
        p.out[(uint64_t)line * p.out_ls + (uint64_t)t * p.out_ts] = v;
    }
}

// ---- host arithmetic (the reference's pow_mod / inverse semantics) ----------

uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)(((unsigned __int128)a * b) % q);
}
// ntt/cpp/ntt.cpp:78-87: r starts at 1, the base is reduced first.
uint64_t h_powmod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1;
    b %= q;
    while (e) {
        if (e & 1) r = h_mulmod(r, b, q);
        b = h_mulmod(b, b, q);
        e >>= 1;
    }
    return r;
}

// Standard-form value -> twiddle representation of the path.
uint64_t h_rep(const WArith& A, uint64_t x) {
    if (A.mode == W_CYC) return (uint64_t)(((unsigned __int128)x << 32) % CYC_Q);
    if (A.even) return x % A.q;
    return (uint64_t)(((unsigned __int128)(x % A.q) << 64) % A.q);
}

WArith make_arith(int mode, uint64_t q) {
    WArith A{};
    A.mode = mode;
    A.q = q;
    A.even = (mode != W_CYC) && !(q & 1);
    if (!A.even && mode != W_CYC) {
        uint64_t x = q;  // Newton: q*x = 1 mod 2^(3*2^k)
        for (int i = 0; i < 5; ++i) x *= 2 - q * x;
        A.qinv = 0 - x;
    }
    return A;
}

uint32_t log2_u(size_t n) {
    uint32_t l = 0;
    while (((size_t)1 << l) < n) ++l;
    return l;
}

}  // namespace

struct WordNttCache {
    struct Tables {
        DevBuf buf;
        uint32_t h = 0;
    };
    std::map<std::tuple<uint32_t, uint64_t, uint64_t, int>, Tables> tables;
    ~WordNttCache() {
        for (auto& kv : tables) kv.second.buf.release();
    }
};

WordNttCache* word_ntt_cache_create() { return new WordNttCache(); }
void word_ntt_cache_destroy(WordNttCache* c) { delete c; }

// Tables lo[k] = w^k (k < 2^h) and hi[k] = w^(k 2^h) (k < 2^(log_n - h)), in
// the path's representation, cached per (n, q, w, representation).
static const WordNttCache::Tables& get_tables(WordNttCache* cache, const WArith& A, uint32_t log_n,
                                              uint64_t w, cudaStream_t st) {
    const int rep = A.mode == W_CYC ? 0 : (A.even ? 2 : 1);
    const auto key = std::make_tuple(log_n, A.q, w, rep);
    auto it = cache->tables.find(key);
    if (it != cache->tables.end()) return it->second;
    if (cache->tables.size() >= 64) {
        KB_CUDA(cudaStreamSynchronize(st));
        for (auto& kv : cache->tables) kv.second.buf.release();
        cache->tables.clear();
    }
    const uint32_t h = (log_n + 1) / 2;
    const size_t nlo = (size_t)1 << h, nhi = (size_t)1 << (log_n - h);
    std::vector<uint64_t> host(nlo + nhi);
    uint64_t cur = 1 % A.q;
    for (size_t k = 0; k < nlo; ++k) {
        host[k] = h_rep(A, cur);
        cur = h_mulmod(cur, w, A.q);
    }
    const uint64_t step = h_powmod(w, nlo, A.q);
    cur = 1 % A.q;
    for (size_t k = 0; k < nhi; ++k) {
        host[nlo + k] = h_rep(A, cur);
        cur = h_mulmod(cur, step, A.q);
    }
    WordNttCache::Tables& T = cache->tables[key];
    T.h = h;
    T.buf.reserve(host.size() * 8, st);
    KB_CUDA(cudaMemcpyAsync(T.buf.ptr, host.data(), host.size() * 8, cudaMemcpyHostToDevice, st));
    KB_CUDA(cudaStreamSynchronize(st));  // the host vector dies here
    return T;
}

static void launch_pass(const WArith& A, WPass p, cudaStream_t st) {
    p.lpc = std::max<uint32_t>(1, WNTT_TILE >> p.log_L);
    const unsigned grid = (p.lines + p.lpc - 1) / p.lpc;
    k_wntt_pass<<<grid, WNTT_THREADS, 0, st>>>(A, p);
    KB_LAUNCH_CHECK();
}

int word_ntt_device(WordNttCache* cache, uint64_t* d_data, uint64_t* d_scratch, size_t n,
                    uint64_t q, uint64_t root, bool inverse, cudaStream_t st) {
    if (!d_data || n == 0 || (n & (n - 1))) return -1;
    const uint32_t log_n = log2_u(n);
    if (n <= ((size_t)1 << CYC_MAX_LOG)) {
        if (q == 0) return -1;
        if (n <= 1) return 0;
        const uint64_t cyc_root_inv = h_powmod(CYC_ROOT, CYC_Q - 2, CYC_Q);
        const bool cyc = q == CYC_Q &&
                         (inverse ? (root == CYC_ROOT || root == cyc_root_inv) : root == CYC_ROOT);
        const WArith A = make_arith(cyc ? W_CYC : W_SMALL, q);
        uint64_t w, scale = 0;
        if (cyc) {
            w = h_powmod(CYC_ROOT, (1ull << CYC_MAX_LOG) >> log_n, CYC_Q);
            if (inverse) w = h_powmod(w, CYC_Q - 2, CYC_Q);
            if (inverse) scale = h_rep(A, h_powmod(n, CYC_Q - 2, CYC_Q));
        } else {
            w = root;  // the n-th root as given (root_inv for the inverse)
            if (inverse) scale = h_rep(A, h_powmod(n, q - 2, q));
        }
        const auto& T = get_tables(cache, A, log_n, w % q, st);
        WPass p{};
        p.log_n = log_n;
        p.tw_lo = T.buf.as<uint64_t>();
        p.tw_hi = p.tw_lo + ((size_t)1 << T.h);
        p.h = T.h;
        p.reduce_in = A.mode == W_SMALL;
        p.bitrev = 1;
        if (log_n <= WNTT_MAX_LINE_LOG) {
            p.in = d_data;
            p.out = d_data;
            p.lines = 1;
            p.log_L = log_n;
            p.in_ls = p.out_ls = n;
            p.in_ts = p.out_ts = 1;
            p.s_lo = 1;
            p.s_hi = log_n;
            p.post = inverse ? 2 : 0;
            p.scale = scale;
            launch_pass(A, p, st);
            return 0;
        }
        if (!d_scratch) return -1;
        // pass 1: the bit-reversed 2^11-element blocks, stages 1..11
        const uint32_t lb = log_n - WNTT_MAX_LINE_LOG;
        p.in = d_data;
        p.out = d_scratch;
        p.lines = 1u << lb;
        p.log_L = WNTT_MAX_LINE_LOG;
        p.in_ls = 1;
        p.in_ts = 1ull << lb;
        p.line_rev_bits = lb;
        p.out_ls = 1ull << WNTT_MAX_LINE_LOG;
        p.out_ts = 1;
        p.s_lo = 1;
        p.s_hi = WNTT_MAX_LINE_LOG;
        launch_pass(A, p, st);
        // pass 2: columns (stride 2^11), stages 12..log_n
        WPass p2 = p;
        p2.in = d_scratch;
        p2.out = d_data;
        p2.lines = 1u << WNTT_MAX_LINE_LOG;
        p2.log_L = lb;
        p2.in_ls = p2.out_ls = 1;
        p2.in_ts = p2.out_ts = 1ull << WNTT_MAX_LINE_LOG;
        p2.line_rev_bits = 0;
        p2.bitrev = 0;
        p2.reduce_in = 0;
        p2.s_lo = WNTT_MAX_LINE_LOG + 1;
        p2.s_hi = log_n;
        p2.gl = 1;
        p2.log_gt = WNTT_MAX_LINE_LOG;
        p2.post = inverse ? 2 : 0;
        p2.scale = scale;
        launch_pass(A, p2, st);
        return 0;
    }
    if (n > ((size_t)1 << LARGE_MAX_LOG)) return -1;
    if (q == 0) return -1;  // 2^64: the even n has no inverse (ntt_large.cpp:66-76)
    const WArith A = make_arith(W_LARGE, q);
    // ntt_large.cpp:174-182: the transform root is omega^2; the inverse
    // recovers the forward 2n-th root by Fermat (c_ntt.cpp:147-160).
    const uint64_t omega = inverse ? h_powmod(root, q - 2, q) : root;
    const uint64_t wn = h_mulmod(omega, omega, q);
    const uint64_t w = inverse ? h_powmod(wn, q - 2, q) : wn;
    const auto& T = get_tables(cache, A, log_n, w, st);
    const uint32_t l1 = log_n / 2, l2 = log_n - l1;
    WPass col{};
    col.in = col.out = d_data;
    col.lines = 1u << l2;
    col.log_L = l1;
    col.in_ls = col.out_ls = 1;
    col.in_ts = col.out_ts = 1ull << l2;
    col.bitrev = 1;
    col.s_lo = 1;
    col.s_hi = l1;
    col.log_n = log_n;
    col.tw_lo = T.buf.as<uint64_t>();
    col.tw_hi = col.tw_lo + ((size_t)1 << T.h);
    col.h = T.h;
    WPass row = col;
    row.lines = 1u << l1;
    row.log_L = l2;
    row.in_ls = row.out_ls = 1ull << l2;
    row.in_ts = row.out_ts = 1;
    row.s_hi = l2;
    if (!inverse) {
        col.post = 1;  // diagonal w^(i*j)
        launch_pass(A, col, st);
        launch_pass(A, row, st);
    } else {
        row.post = 1;
        launch_pass(A, row, st);
        col.post = 2;
        col.scale = h_rep(A, h_powmod(n, q - 2, q));
        launch_pass(A, col, st);
    }
    return 0;
}

}  // namespace kb200
