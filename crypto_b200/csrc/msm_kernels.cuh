// Curve-templated MSM kernels.  Included by msm_bls.cu and msm_bn.cu, which
// instantiate one launcher table each (so the two curves compile in
// parallel); the host driver in msm.cu only sees MsmLaunchers.
#pragma once
#include "curve.cuh"
#include "msm_desc.cuh"
#include "runtime.cuh"

namespace kb200 {


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

// GLV split for BLS12-381 G1: with u = -0xd201000000010000 the curve
// parameter, lambda = u^2 - 1 (128 bits) is a cube root of unity mod r and
// phi(x, y) = (beta2 x, y), beta2 a cube root of unity mod p, acts on G1 as
// [lambda].  A scalar k < r = lambda^2 + lambda + 1 splits as
// k = k1 + k2 lambda with k1 = k mod lambda and k2 = k div lambda, both
// below 2^128, so k P = k1 P + k2 phi(P): twice the points, half the
// windows.  The quotient comes from Barrett reduction with
// mu = floor(2^384 / lambda) (exact for k < r; a correction loop covers the
// bound).  Little-endian 32-bit words.
static __constant__ uint32_t kGlvLambda[4] = {0xffffffff, 0x00000000, 0x0001a402, 0xac45a401};
static __constant__ uint32_t kGlvMu[9] = {0x896c72dd, 0xda5e4f8d, 0x268bf7a3, 0x389f49a7, 0xf6cfee30,
                                   0x63f6e522, 0xe01faadd, 0x7c6becf1, 0x00000001};
// 2^256 mod r: the reference's dropped top carry subtracts 2^256.
static __constant__ uint32_t kR256ModR[8] = {0xfffffffe, 0x00000001, 0x00034802, 0x5884b7fa,
                                      0xecbc4ff5, 0x998c4fef, 0xacc5056f, 0x1824b159};

__device__ __forceinline__ bool geq_words(const uint32_t* a, const uint32_t* b, int n) {
    for (int i = n - 1; i >= 0; --i)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}
__device__ __forceinline__ void sub_words(uint32_t* a, const uint32_t* b, int n) {
    uint32_t br = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t d = (uint64_t)a[i] - b[i] - br;
        a[i] = (uint32_t)d;
        br = (uint32_t)(d >> 63);
    }
}

// k (8 words, < r) -> k1 = k mod lambda, k2 = k div lambda (4 words each).
static __device__ void glv_split(const uint32_t k[8], uint32_t k1[4], uint32_t k2[4]) {
    uint32_t prod[17];
    for (int i = 0; i < 17; ++i) prod[i] = 0;
    for (int i = 0; i < 8; ++i) {
        uint64_t carry = 0;
        for (int j = 0; j < 9; ++j) {
            const uint64_t t = (uint64_t)k[i] * kGlvMu[j] + prod[i + j] + carry;
            prod[i + j] = (uint32_t)t;
            carry = t >> 32;
        }
        prod[i + 9] = (uint32_t)carry;
    }
    uint32_t q[5];
    for (int i = 0; i < 5; ++i) q[i] = prod[12 + i];  // floor(k mu / 2^384)
    // rem = k - q lambda (fits: 0 <= rem < 2^129 before correction)
    uint32_t ql[9];
    for (int i = 0; i < 9; ++i) ql[i] = 0;
    for (int i = 0; i < 5; ++i) {
        uint64_t carry = 0;
        for (int j = 0; j < 4; ++j) {
            const uint64_t t = (uint64_t)q[i] * kGlvLambda[j] + ql[i + j] + carry;
            ql[i + j] = (uint32_t)t;
            carry = t >> 32;
        }
        if (i + 4 < 9) ql[i + 4] = (uint32_t)carry;
    }
    uint32_t rem[8];
    for (int i = 0; i < 8; ++i) rem[i] = k[i];
    sub_words(rem, ql, 8);
    uint32_t lam8[8] = {kGlvLambda[0], kGlvLambda[1], kGlvLambda[2], kGlvLambda[3], 0, 0, 0, 0};
    for (int guard = 0; guard < 4 && geq_words(rem, lam8, 8); ++guard) {
        sub_words(rem, lam8, 8);
        uint32_t c = 1;
        for (int i = 0; i < 5 && c; ++i) {
            q[i] += c;
            c = q[i] == 0;
        }
    }
    for (int i = 0; i < 4; ++i) {
        k1[i] = rem[i];
        k2[i] = q[i];
    }
}

// GLV split for BN254 G1 (Gallant-Lambert-Vanstone, CRYPTO 2001, with
// Babai rounding): the lattice {(x, y) : x + y lambda = 0 mod r} has the
// reduced basis v1 = (a1, -b1), v2 = (a2, b2) (extended Euclid on (r,
// lambda), det = r), a1 = b2 = 0x89d3256894d213e3,
// b1 = 0x6f4d8248eeb859fc8211bbeb7d4f1128, a2 = 0x6f4d8248eeb859fd0be4e1541221250b.
// With cA = round(k b2 / r), cB = round(k b1 / r) -- each computed as
// (k g + 2^383) >> 384, g = round(2^384 b / r) --
//   k1 = k - cA a1 - cB a2,   k2 = cA b1 - cB b2,
// so k1 + k2 lambda = k (mod r) exactly and |k1|, |k2| < 2^126 for every
// k < r.  The halves are signed: their signs go to the entries' sign bits.
static __constant__ uint32_t kBnGlvG2[7] = {0x2fafba64, 0x8fa7d32d, 0x773a6ef2, 0x6eb9c714,
                                            0xc7e0b3d7, 0xd91d232e, 0x00000002};
static __constant__ uint32_t kBnGlvG1[9] = {0x9b9bdffa, 0x86937516, 0x5eaa26d9, 0xa5e38cfb, 0x391eb18d,
                                            0x7a7bd9d4, 0xa773d2cf, 0x4ccef014, 0x00000002};
static __constant__ uint32_t kBnGlvA1[2] = {0x94d213e3, 0x89d32568};
static __constant__ uint32_t kBnGlvB1[4] = {0x7d4f1128, 0x8211bbeb, 0xeeb859fc, 0x6f4d8248};
static __constant__ uint32_t kBnGlvA2[4] = {0x1221250b, 0x0be4e154, 0xeeb859fd, 0x6f4d8248};
static __constant__ uint32_t kBnGlvB2[2] = {0x94d213e3, 0x89d32568};
// 2^256 mod r (BN254): the reference's dropped top carry subtracts 2^256.
static __constant__ uint32_t kBnR256ModR[8] = {0x4ffffffb, 0xac96341c, 0x9f60cd29, 0x36fc7695,
                                               0x7879462e, 0x666ea36f, 0x9a07df2f, 0x0e0a77c1};

// round(k g / 2^384) for k of 8 words and g of ng <= 9 words: nr words out.
static __device__ void mul_round384(const uint32_t k[8], const uint32_t* g, int ng, uint32_t* out,
                                    int nr) {
    uint32_t prod[17];
    for (int i = 0; i < 17; ++i) prod[i] = 0;
    for (int i = 0; i < 8; ++i) {
        uint64_t carry = 0;
        for (int j = 0; j < ng; ++j) {
            const uint64_t t = (uint64_t)k[i] * g[j] + prod[i + j] + carry;
            prod[i + j] = (uint32_t)t;
            carry = t >> 32;
        }
        prod[i + ng] = (uint32_t)carry;
    }
    // + 2^383 (bit 31 of word 11), then the words from 12 up
    uint64_t cy = (uint64_t)prod[11] + 0x80000000u;
    prod[11] = (uint32_t)cy;
    cy >>= 32;
    for (int i = 12; i < 17; ++i) {
        cy += prod[i];
        prod[i] = (uint32_t)cy;
        cy >>= 32;
    }
    for (int i = 0; i < nr; ++i) out[i] = prod[12 + i];
}

// acc (8 words, two's complement) += sgn * (a (na words) * b (nb words)).
static __device__ void mac_signed(uint32_t acc[8], const uint32_t* a, int na, const uint32_t* b,
                                  int nb, bool subtract) {
    uint32_t t[8];
    for (int i = 0; i < 8; ++i) t[i] = 0;
    for (int i = 0; i < na; ++i) {
        uint64_t carry = 0;
        for (int j = 0; j < nb && i + j < 8; ++j) {
            const uint64_t v = (uint64_t)a[i] * b[j] + t[i + j] + carry;
            t[i + j] = (uint32_t)v;
            carry = v >> 32;
        }
        if (i + nb < 8) t[i + nb] = (uint32_t)carry;
    }
    if (subtract) {
        sub_words(acc, t, 8);
    } else {
        uint64_t cy = 0;
        for (int i = 0; i < 8; ++i) {
            cy += (uint64_t)acc[i] + t[i];
            acc[i] = (uint32_t)cy;
            cy >>= 32;
        }
    }
}

// Two's complement (8 words) -> magnitude (4 words) and sign.
static __device__ void signed_to_mag(const uint32_t v[8], uint32_t mag[4], uint32_t& neg) {
    neg = v[7] >> 31;
    uint32_t cy = neg;
    for (int i = 0; i < 4; ++i) {
        const uint64_t x = (uint64_t)(neg ? ~v[i] : v[i]) + cy;
        mag[i] = (uint32_t)x;
        cy = (uint32_t)(x >> 32);
    }
}

// k (8 words, < r) -> |k1|, |k2| (4 words each) and their signs.
static __device__ void glv_split_bn(const uint32_t k[8], uint32_t k1[4], uint32_t k2[4],
                                    uint32_t& neg1, uint32_t& neg2) {
    uint32_t cA[2], cB[4];
    mul_round384(k, kBnGlvG2, 7, cA, 2);
    mul_round384(k, kBnGlvG1, 9, cB, 4);
    uint32_t a1[2] = {kBnGlvA1[0], kBnGlvA1[1]};
    uint32_t a2[4] = {kBnGlvA2[0], kBnGlvA2[1], kBnGlvA2[2], kBnGlvA2[3]};
    uint32_t b1[4] = {kBnGlvB1[0], kBnGlvB1[1], kBnGlvB1[2], kBnGlvB1[3]};
    uint32_t b2[2] = {kBnGlvB2[0], kBnGlvB2[1]};
    uint32_t s1[8], s2[8];
    for (int i = 0; i < 8; ++i) {
        s1[i] = k[i];
        s2[i] = 0;
    }
    mac_signed(s1, cA, 2, a1, 2, true);
    mac_signed(s1, cB, 4, a2, 4, true);
    mac_signed(s2, cA, 2, b1, 4, false);
    mac_signed(s2, cB, 4, b2, 2, true);
    signed_to_mag(s1, k1, neg1);
    signed_to_mag(s2, k2, neg2);
}

// Signed-digit recoding, one thread per scalar of the batch.  Entry (w, j)
// of item i lives at entry_base_i + w * n_i + j (GLV items: k1's digit at
// entry_base_i + w * 2 n_i + j, k2's at entry_base_i + w * 2 n_i + n_i + j).
// quirk_c: 0, or the reference window size (4 or 8) whose dropped top carry
// is reproduced by negating (s, P) -> (2^256 - s, -P) for s above the
// carry threshold 0x8888...88 (c = 4) or 0x8080...80 (c = 8).
template <class C>
__global__ void k_recode(const ItemDesc* __restrict__ items, uint32_t n_items,
                         unsigned long long first, unsigned long long count,
                         const uint32_t* __restrict__ scalars,
                         const uint32_t* __restrict__ table, uint32_t* __restrict__ keys,
                         uint32_t* __restrict__ vals) {
    using F = typename C::F;
    const unsigned long long idx = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    const unsigned long long g = first + idx;  // scalar index over all items
    // item: largest i with items[i].scalar_off <= g
    uint32_t lo = 0, hi = n_items;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (items[mid].scalar_off <= g)
            lo = mid;
        else
            hi = mid;
    }
    const ItemDesc it = items[lo];
    if (g < it.scalar_off || g - it.scalar_off >= it.n) return;  // gap between items
    const uint32_t j = (uint32_t)(g - it.scalar_off);
    const uint32_t row = it.point_off + j;
    // Without a table (points still in flight) infinity points get entries
    // too: every later stage skips infinity rows.
    const bool inf = table && aff_is_inf_words<F>(table + (size_t)row * 2 * F::N);
    uint32_t s[8];
    const uint4* sp = reinterpret_cast<const uint4*>(scalars + g * 8);
    const uint4 a = sp[0], b = sp[1];
    s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
    s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
    uint32_t neg = 0;
    bool dropped_carry = false;
    if (it.quirk_c == 4 || it.quirk_c == 8) {
        const uint32_t t = it.quirk_c == 4 ? 0x88888888u : 0x80808080u;
        int gt = 0;
#pragma unroll
        for (int k = 7; k >= 0; --k) {
            if (gt == 0) {
                if (s[k] > t) gt = 1;
                else if (s[k] < t) gt = -1;
            }
        }
        dropped_carry = gt == 1;
    }
    const int c = (int)it.c;
    const uint32_t M = it.M;
    const uint32_t mask = (1u << c) - 1u;
    // Signed digits of the nw-word scalar sc over the item's W windows; the
    // digit of window w goes to entry slot0 + w * wstride with point row prow.
    auto emit = [&](const uint32_t* sc, int nw, uint32_t prow, unsigned long long slot0,
                    unsigned long long wstride, uint32_t negbit) {
        uint32_t carry = 0;
        for (int w = 0; w < (int)it.W; ++w) {
            const int off = w * c;
            const int wd = off >> 5, sh = off & 31;
            uint32_t raw = 0;
            if (wd < nw) {
                const uint64_t lo64 = sc[wd];
                const uint64_t hi64 = (wd + 1 < nw) ? sc[wd + 1] : 0;
                raw = (uint32_t)(((hi64 << 32) | lo64) >> sh) & mask;
            }
            uint32_t d = raw + carry;
            uint32_t sign = 0;
            // a GLV half's top window stays unsigned: nothing carries past it
            if (d > M && !(it.glv && w == (int)it.W - 1)) {
                d = (1u << c) - d;
                sign = 1;
                carry = 1;
            } else {
                carry = 0;
            }
            const unsigned long long slot = slot0 + (unsigned long long)w * wstride;
            if (d == 0 || inf) {
                keys[slot] = KEY_SENTINEL;
            } else if (it.chunk_rows) {
                keys[slot] = (j / it.chunk_rows) * it.chunk_stride + it.bucket_base +
                             (uint32_t)w * M + (d - 1);
                vals[slot] = prow | ((sign ^ negbit) << 31);
            } else if (it.row_stride) {
                // shifted table: level w holds 2^(c*w) times the point, so every
                // window feeds the same buckets
                keys[slot] = it.bucket_base + (d - 1);
                vals[slot] = (prow + (uint32_t)w * it.row_stride) | ((sign ^ negbit) << 31);
            } else {
                keys[slot] = it.bucket_base + (uint32_t)w * M + (d - 1);
                vals[slot] = prow | ((sign ^ negbit) << 31);
            }
        }
    };
    if constexpr (C::CURVE_ID == 2) {
        if (it.glv) {
            // k = s mod r (s < 2^256 < 3r), minus 2^256 where the reference
            // drops its top carry
            uint32_t k[8], r8[8];
            for (int i = 0; i < 8; ++i) {
                k[i] = s[i];
                r8[i] = FrBLS::P(i);
            }
            for (int guard = 0; guard < 3 && geq_words(k, r8, 8); ++guard) sub_words(k, r8, 8);
            if (dropped_carry) {
                uint32_t t[8];
                for (int i = 0; i < 8; ++i) t[i] = kR256ModR[i];
                if (geq_words(k, t, 8)) {
                    sub_words(k, t, 8);
                } else {  // k + r - t
                    uint64_t cy = 0;
                    for (int i = 0; i < 8; ++i) {
                        cy += (uint64_t)k[i] + r8[i];
                        k[i] = (uint32_t)cy;
                        cy >>= 32;
                    }
                    sub_words(k, t, 8);
                }
            }
            uint32_t k1[4], k2[4];
            glv_split(k, k1, k2);
            const unsigned long long base = it.entry_base + j;
            emit(k1, 4, row, base, 2ull * it.n, 0u);
            emit(k2, 4, row + it.glv_off, base + it.n, 2ull * it.n, 0u);
            return;
        }
    }
    if constexpr (C::CURVE_ID == 1) {
        if (it.glv) {
            // k = s mod r (s < 2^256 < 6r), minus 2^256 where the reference
            // drops its top carry; signed halves, signs into the entries
            uint32_t k[8], r8[8];
            for (int i = 0; i < 8; ++i) {
                k[i] = s[i];
                r8[i] = FrBN::P(i);
            }
            for (int guard = 0; guard < 6 && geq_words(k, r8, 8); ++guard) sub_words(k, r8, 8);
            if (dropped_carry) {
                uint32_t t[8];
                for (int i = 0; i < 8; ++i) t[i] = kBnR256ModR[i];
                if (geq_words(k, t, 8)) {
                    sub_words(k, t, 8);
                } else {  // k + r - t
                    uint64_t cy = 0;
                    for (int i = 0; i < 8; ++i) {
                        cy += (uint64_t)k[i] + r8[i];
                        k[i] = (uint32_t)cy;
                        cy >>= 32;
                    }
                    sub_words(k, t, 8);
                }
            }
            uint32_t k1[4], k2[4], n1, n2;
            glv_split_bn(k, k1, k2, n1, n2);
            const unsigned long long base = it.entry_base + j;
            emit(k1, 4, row, base, 2ull * it.n, n1);
            emit(k2, 4, row + it.glv_off, base + it.n, 2ull * it.n, n2);
            return;
        }
    }
    if (dropped_carry) {
        uint32_t cy = 1;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint64_t v = (uint64_t)(~s[k]) + cy;
            s[k] = (uint32_t)v;
            cy = (uint32_t)(v >> 32);
        }
        neg = 1;
    }
    emit(s, 8, row, it.entry_base + j, (unsigned long long)it.n, neg);
}

// Wire points (big-endian x || y, all-zero = infinity) -> table rows, read
// in 16-byte pieces when the wire base is 16-byte aligned (rows are 64 or
// 96 bytes), byte by byte otherwise.  glv_stride: 0, or the row distance of
// the GLV rows: row i + glv_stride gets phi(P_i) = (beta x, y) (beta2 on
// BLS12-381).
template <class C, bool V16>
__global__ void k_wire_to_table(const uint8_t* __restrict__ wire, uint32_t* __restrict__ table,
                                size_t n, size_t glv_stride) {
    using F = typename C::F;
    constexpr int N = F::N;
    static_assert(C::WIRE == 8 * N, "wire row = two N-word coordinates");
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t m[2 * N];  // the row's 4-byte groups in memory order
    if constexpr (V16) {
        const uint4* s = reinterpret_cast<const uint4*>(wire + i * C::WIRE);
#pragma unroll
        for (int k = 0; k < N / 2; ++k) {
            const uint4 v = s[k];
            m[4 * k] = v.x;
            m[4 * k + 1] = v.y;
            m[4 * k + 2] = v.z;
            m[4 * k + 3] = v.w;
        }
    } else {
        const uint8_t* w = wire + i * C::WIRE;
#pragma unroll
        for (int q = 0; q < 2 * N; ++q)
            m[q] = (uint32_t)w[4 * q] | ((uint32_t)w[4 * q + 1] << 8) | ((uint32_t)w[4 * q + 2] << 16) |
                   ((uint32_t)w[4 * q + 3] << 24);
    }
    uint32_t any = 0;
#pragma unroll
    for (int q = 0; q < 2 * N; ++q) any |= m[q];
    uint32_t* dst = table + i * 2 * N;
    Fe<F> x, y;
    if (!any) {
        fe_zero(x);
        fe_zero(y);
        x.v[N - 1] = INF_FLAG;
        fe_store16(dst, x);
        fe_store16(dst + N, y);
        if (glv_stride) {
            fe_store16(dst + glv_stride * 2 * N, x);
            fe_store16(dst + glv_stride * 2 * N + N, y);
        }
        return;
    }
    // limb l (little-endian words) = the big-endian group N - 1 - l, bytes swapped
#pragma unroll
    for (int l = 0; l < N; ++l) {
        x.v[l] = __byte_perm(m[N - 1 - l], 0, 0x0123);
        y.v[l] = __byte_perm(m[2 * N - 1 - l], 0, 0x0123);
    }
    fe_to_mont(x, x);
    fe_to_mont(y, y);
    fe_store16(dst, x);
    fe_store16(dst + N, y);
    if (glv_stride) {
        Fe<F> b;
#pragma unroll
        for (int k = 0; k < N; ++k) b.v[k] = C::CURVE_ID == 2 ? kGlvBeta2Mont[k] : kBnGlvBetaMont[k % 8];
        fe_mul(x, x, b);
        fe_store16(dst + glv_stride * 2 * N, x);
        fe_store16(dst + glv_stride * 2 * N + N, y);
    }
}


template <class F>
__device__ __forceinline__ void load_table_point(Affine<F>& a, const uint32_t* table, uint32_t idx) {
    const uint4* src = reinterpret_cast<const uint4*>(table + (size_t)idx * 2 * F::N);
    uint32_t w[2 * F::N];
#pragma unroll
    for (int k = 0; k < F::N / 2; ++k) {
        const uint4 v = src[k];
        w[4 * k] = v.x;
        w[4 * k + 1] = v.y;
        w[4 * k + 2] = v.z;
        w[4 * k + 3] = v.w;
    }
    aff_load(a, w);
}

// Bucket holding sorted entry e: the largest b with offsets[b] <= e (empty
// buckets share their successor's offset, so the largest one is the
// non-empty bucket that owns e).
__device__ __forceinline__ uint32_t bucket_of(const uint32_t* offsets, uint32_t B, uint32_t e) {
    uint32_t lo = 0, hi = B;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (offsets[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Level 1, persistent: CTAs pull units of blockDim.x chunks from *queue.
// Lane t sums chunk t = entries [tK, tK + K) of the bucket-sorted list
// with mixed XYZZ additions, flushing at bucket boundaries: the run of the
// chunk's first bucket goes to rec_first[t], the run of its last bucket (if
// different) to rec_last[t], runs of buckets strictly inside the chunk
// straight to buckets[].  Every lane does exactly K additions (the last
// chunk fewer), whatever the bucket sizes.
// The running sum lives in shared memory (SmXyzz), so registers hold only
// the formula's temporaries and more warps stay resident to hide the
// latency of the dependent multiply chains.
template <class C>
__global__ void __launch_bounds__(128, C::ACC_MIN_BLOCKS) k_accumulate(AccArgs a) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;
    __shared__ uint32_t unit;
    __shared__ uint32_t s_acc[4 * F::N * 128];
    const SmXyzz<F, 128> acc{s_acc + threadIdx.x};
    // Only non-zero digits were sorted: the list length is offsets[B].
    const uint32_t L = a.offsets[a.B];
    const uint32_t nchunks = (L + a.K - 1) / a.K;
    for (;;) {
        if (threadIdx.x == 0) unit = atomicAdd(a.queue, 1u);
        __syncthreads();
        const uint32_t base = unit * blockDim.x;
        __syncthreads();
        if (base >= nchunks) return;
        const uint32_t t = base + threadIdx.x;
        if (t < nchunks) {
            const uint32_t e0 = t * a.K;
            const uint32_t e1 = min(e0 + a.K, L);
            uint32_t b = bucket_of(a.offsets, a.B, e0);
            uint32_t bend = a.offsets[b + 1];
            uint32_t run0 = e0;
            acc.set_inf();
            uint32_t v = a.sorted ? a.sorted[e0] : e0;
            for (uint32_t e = e0; e < e1; ++e) {
                if (e == bend) {
                    // flush the finished run [run0, e) of bucket b
                    uint32_t* dst = (run0 == e0) ? a.rec_first + (size_t)t * PW
                                                 : a.buckets + (size_t)b * PW;
                    acc.to_global(dst);
                    acc.set_inf();
                    while (a.offsets[b + 1] <= e) ++b;
                    bend = a.offsets[b + 1];
                    run0 = e;
                }
                const uint32_t vn = (e + 1 < e1) ? (a.sorted ? a.sorted[e + 1] : e + 1) : 0u;
                if (e + 1 < e1) {
                    const uint32_t* nxt = a.table + (size_t)(vn & 0x7fffffffu) * 2 * F::N;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(nxt));
                }
                const uint32_t* row = a.table + (size_t)(v & 0x7fffffffu) * 2 * F::N;
                if (!aff_is_inf_words<F>(row)) {  // pairing levels can produce infinity
                    Affine<F> p;
                    load_table_point<F>(p, a.table, v & 0x7fffffffu);
                    if (v >> 31) fe_neg(p.y, p.y);
                    xyzz_add_affine(acc, p);
                }
                v = vn;
            }
            uint32_t* dst = (run0 == e0) ? a.rec_first + (size_t)t * PW : a.rec_last + (size_t)t * PW;
            acc.to_global(dst);
        }
    }
}

// ---- Batch-affine pairing levels -------------------------------------------
// One level halves every bucket's run: slot k of bucket b adds input points
// i0 = in_off[b] + 2 (k - out_off[b]) and i0 + 1 (if still in the run) in
// affine coordinates,
//   lambda = (y1 - y0) / (x1 - x0)  (or 3 x0^2 / 2 y0 when the points are
//   equal), x3 = lambda^2 - x0 - x1, y3 = lambda (x0 - x3) - y0,
// with infinity where they cancel.  The denominators are inverted together
// (Montgomery's trick, one field inversion per block of k_inv_wide):
//   k_pair_fwd   thread t owns slots [PAIR_J t, PAIR_J t + PAIR_J): running
//                products of its denominators (prefixes to HBM), total to tot[t];
//   k_inv_wide   every total replaced by its inverse: blocks of INV_T
//                threads, each thread chaining up to INV_G totals, warp-shuffle
//                prefix/suffix products over threads and over warps, one
//                inversion per block;
//   k_pair_bwd   per thread, backwards over its slots: the slot's inverse from
//                its prefix, then the affine sum.
// Per addition: 1 product forward, 2 to recover the inverse, 3 for the sum,
// plus about 4/PAIR_J for the totals' inversion, against 10 for a mixed XYZZ
// addition.  Field
// elements in the scratch arrays are stored word-major (word q of element e
// at q * stride + e) so that consecutive threads touch consecutive words.
enum PairCase : int { PAIR_PASS0 = 0, PAIR_PASS1 = 1, PAIR_INF = 2, PAIR_ADD = 3, PAIR_DBL = 4 };

template <class F>
__device__ __forceinline__ void fe_load_wm(Fe<F>& x, const uint32_t* v, size_t stride, size_t e) {
#pragma unroll
    for (int q = 0; q < F::N; ++q) x.v[q] = v[(size_t)q * stride + e];
}
template <class F>
__device__ __forceinline__ void fe_store_wm(uint32_t* v, size_t stride, size_t e, const Fe<F>& x) {
#pragma unroll
    for (int q = 0; q < F::N; ++q) v[(size_t)q * stride + e] = x.v[q];
}

// Rows of the two operands of input position i (level 0: a table row by
// sorted index, sign in bit 31; later levels: the previous level's rows).
template <class F>
__device__ __forceinline__ const uint32_t* pair_row(const PairArgs& a, uint32_t i, bool& neg) {
    if (a.sorted) {
        const uint32_t v = a.sorted[i];
        neg = (v >> 31) != 0;
        return a.src + (size_t)(v & 0x7fffffffu) * 2 * F::N;
    }
    neg = false;
    return a.src + (size_t)i * 2 * F::N;
}

// W consecutive words (W a multiple of 4, src and dst 16-byte aligned: rows
// are 2N words and N is a multiple of 4) in 16-byte accesses.
template <int W>
__device__ __forceinline__ void ld_words16(uint32_t* w, const uint32_t* src) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
    for (int k = 0; k < W / 4; ++k) {
        const uint4 v = s[k];
        w[4 * k] = v.x;
        w[4 * k + 1] = v.y;
        w[4 * k + 2] = v.z;
        w[4 * k + 3] = v.w;
    }
}
template <int W>
__device__ __forceinline__ void st_words16(uint32_t* dst, const uint32_t* w) {
    uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int k = 0; k < W / 4; ++k) d[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
}

template <class F>
__device__ __forceinline__ void pair_load(const PairArgs& a, uint32_t i, Affine<F>& P, bool& inf) {
    bool neg;
    const uint32_t* row = pair_row<F>(a, i, neg);
    uint32_t w[2 * F::N];
    ld_words16<2 * F::N>(w, row);
    inf = aff_is_inf_words<F>(w);
    aff_load(P, w);
    if (neg) fe_neg(P.y, P.y);
}

// Output row of a pairing slot: affine (x, y), or the infinity flag.
template <class F>
__device__ __forceinline__ void pair_store(uint32_t* dst, const Fe<F>& x, const Fe<F>& y) {
    uint32_t w[2 * F::N];
#pragma unroll
    for (int q = 0; q < F::N; ++q) {
        w[q] = x.v[q];
        w[F::N + q] = y.v[q];
    }
    st_words16<2 * F::N>(dst, w);
}

// Loads slot k's operands (bucket b) and classifies it; den is the
// denominator that joins the batch inversion (one for the non-additions).
template <class F>
__device__ __forceinline__ int pair_setup(const PairArgs& a, uint32_t k, uint32_t b, Affine<F>& P0,
                                          Affine<F>& P1, bool& inf0, Fe<F>& den) {
    const uint32_t i0 = a.in_off[b] + 2 * (k - a.out_off[b]);
    const bool has1 = i0 + 1 < a.in_off[b + 1];
    bool inf1 = true;
    pair_load<F>(a, i0, P0, inf0);
    if (has1) pair_load<F>(a, i0 + 1, P1, inf1);
    fe_one(den);
    if (inf1) return PAIR_PASS0;
    if (inf0) return PAIR_PASS1;
    if (!fe_eq(P0.x, P1.x)) {
        fe_sub(den, P1.x, P0.x);
        return PAIR_ADD;
    }
    if (fe_eq(P0.y, P1.y) && !fe_is_zero(P0.y)) {
        fe_dbl(den, P0.y);
        return PAIR_DBL;
    }
    return PAIR_INF;
}

// Only the denominator of slot k: the x coordinates, and the y coordinates
// when the x are equal.  Matches pair_setup's den in every case.
template <class F>
__device__ __forceinline__ void pair_den(const PairArgs& a, uint32_t k, uint32_t b, Fe<F>& den) {
    fe_one(den);
    const uint32_t i0 = a.in_off[b] + 2 * (k - a.out_off[b]);
    if (i0 + 1 >= a.in_off[b + 1]) return;
    bool n0, n1;
    const uint32_t* r0 = pair_row<F>(a, i0, n0);
    const uint32_t* r1 = pair_row<F>(a, i0 + 1, n1);
    Fe<F> x0, x1;
    ld_words16<F::N>(x0.v, r0);
    ld_words16<F::N>(x1.v, r1);
    if (aff_is_inf_words<F>(x0.v) || aff_is_inf_words<F>(x1.v)) return;
    if (!fe_eq(x0, x1)) {
        fe_sub(den, x1, x0);
        return;
    }
    Fe<F> y0, y1;
    fe_load(y0, r0 + F::N);
    fe_load(y1, r1 + F::N);
    if (n0) fe_neg(y0, y0);
    if (n1) fe_neg(y1, y1);
    if (fe_eq(y0, y1) && !fe_is_zero(y0)) fe_dbl(den, y0);
}

template <class C>
__global__ void __launch_bounds__(256) k_pair_fwd(PairArgs a, uint32_t T, uint32_t* __restrict__ pre,
                                                  uint32_t* __restrict__ tot) {
    using F = typename C::F;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const uint32_t total = a.out_off[a.B];  // slots out_off[0] .. out_off[B]
    const uint32_t k0 = a.out_off[0] + t * (uint32_t)PAIR_J;
    Fe<F> run;
    fe_one(run);
    if (k0 < total) {
        const uint32_t kend = min(k0 + (uint32_t)PAIR_J, total);
        uint32_t b = bucket_of(a.out_off, a.B, k0);
        for (uint32_t k = k0; k < kend; ++k) {
            while (a.out_off[b + 1] <= k) ++b;
            Fe<F> den;
            pair_den<F>(a, k, b, den);
            fe_mul(run, run, den);
            if (k + 1 < kend) fe_store_wm(pre + (size_t)(k - k0) * F::N * T, T, t, run);
        }
    }
    fe_store_wm(tot, T, t, run);  // one for threads without slots
}

template <class C, bool DST_OFF>
__global__ void __launch_bounds__(256, 2) k_pair_bwd(PairArgs a, uint32_t T, const uint32_t* __restrict__ pre,
                                                     const uint32_t* __restrict__ inv_tot) {
    using F = typename C::F;
    constexpr int N = F::N;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const uint32_t total = a.out_off[a.B];
    const uint32_t k0 = a.out_off[0] + t * (uint32_t)PAIR_J;
    if (k0 >= total) return;
    const uint32_t kend = min(k0 + (uint32_t)PAIR_J, total);
    Fe<F> inv_run;
    fe_load_wm(inv_run, inv_tot, T, t);
    uint32_t bend = bucket_of(a.out_off, a.B, kend - 1);
    for (int j = (int)(kend - k0) - 1; j >= 0; --j) {
        const uint32_t k = k0 + (uint32_t)j;
        while (a.out_off[bend] > k) --bend;
        Affine<F> P0, P1;
        bool inf0;
        Fe<F> den, inv;
        const int kind = pair_setup<F>(a, k, bend, P0, P1, inf0, den);
        if (j > 0) {
            fe_load_wm(inv, pre + (size_t)(j - 1) * N * T, T, t);
            // two independent products, inlined so their instruction streams
            // interleave (pair stage at 2^22: 22.65 -> 21.64 ms; inlining the
            // sum's three dependent products as well was slower, 22.47 ms)
            fe_mul_inl(inv, inv, inv_run);
            fe_mul_inl(inv_run, inv_run, den);
        } else {
            inv = inv_run;
        }
        uint32_t row = k;
        if constexpr (DST_OFF) row = a.dst_off[bend] + (k - a.out_off[bend]);
        uint32_t* dst = a.dst + (size_t)row * 2 * N;
        if (kind == PAIR_ADD || kind == PAIR_DBL) {
            Fe<F> lam, x3;
            if (kind == PAIR_ADD) {
                fe_sub(lam, P1.y, P0.y);
            } else {
                fe_sqr(lam, P0.x);
                fe_dbl(x3, lam);
                fe_add(lam, lam, x3);  // 3 x0^2
                P1.x = P0.x;
            }
            fe_mul(lam, lam, inv);
            fe_sqr(x3, lam);
            fe_sub(x3, x3, P0.x);
            fe_sub(x3, x3, P1.x);
            fe_sub(P1.y, P0.x, x3);
            fe_mul(P1.y, lam, P1.y);
            fe_sub(P1.y, P1.y, P0.y);
            pair_store<F>(dst, x3, P1.y);
        } else if (kind == PAIR_INF || (kind == PAIR_PASS0 && inf0)) {
            Fe<F> z;
            fe_zero(z);
            P0.x = z;
            P0.x.v[N - 1] = INF_FLAG;
            pair_store<F>(dst, P0.x, z);
        } else {
            const Affine<F>& R = kind == PAIR_PASS0 ? P0 : P1;
            pair_store<F>(dst, R.x, R.y);
        }
    }
}

// Inclusive prefix P and suffix S products of the warp's values.
template <class F>
__device__ __forceinline__ void warp_prefix_suffix(Fe<F>& P, Fe<F>& S, int lane) {
    Fe<F> o;
    for (int d = 1; d < 32; d <<= 1) {  // inclusive prefix P and suffix S over the warp
#pragma unroll
        for (int q = 0; q < F::N; ++q) o.v[q] = __shfl_up_sync(0xffffffffu, P.v[q], d);
        if (lane >= d) fe_mul(P, P, o);
#pragma unroll
        for (int q = 0; q < F::N; ++q) o.v[q] = __shfl_down_sync(0xffffffffu, S.v[q], d);
        if (lane + d < 32) fe_mul(S, S, o);
    }
}

// r *= P_{lane-1} * S_{lane+1}: the product of the warp's other lanes' values.
template <class F>
__device__ __forceinline__ void warp_exclude_self(Fe<F>& r, const Fe<F>& P, const Fe<F>& S, int lane) {
    Fe<F> o;
#pragma unroll
    for (int q = 0; q < F::N; ++q) o.v[q] = __shfl_up_sync(0xffffffffu, P.v[q], 1);
    if (lane > 0) fe_mul(r, r, o);
#pragma unroll
    for (int q = 0; q < F::N; ++q) o.v[q] = __shfl_down_sync(0xffffffffu, S.v[q], 1);
    if (lane < 31) fe_mul(r, r, o);
}

// The M elements of v (word-major, stride M) replaced by their inverses.
// Block b owns elements [b G INV_T, (b + 1) G INV_T); its thread t chains
// elements base + j INV_T (j < G, base = b G INV_T + t; running products in
// pre, word-major with stride TT = gridDim.x INV_T), the thread products
// combine by warp-shuffle prefix and suffix products, warp 0 repeats that over
// the warp products and its lane 0 inverts the block's product, so every
// thread recovers the inverse of its own product and walks its chain back.
// Elements are non-zero: every denominator is a difference of distinct x, or
// 2y with y non-zero, or one.
template <class F>
__global__ void __launch_bounds__(INV_T, 2) k_inv_wide(uint32_t* __restrict__ v, uint32_t M, uint32_t G,
                                                       uint32_t* __restrict__ pre) {
    constexpr int N = F::N;
    constexpr int NW = INV_T / 32;
    __shared__ uint32_t s_wt[NW * N];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const size_t TT = (size_t)gridDim.x * INV_T;
    const size_t gt = (size_t)blockIdx.x * INV_T + (size_t)t;
    const size_t base = (size_t)blockIdx.x * INV_T * G + (size_t)t;
    Fe<F> run, x;
    fe_one(run);
    uint32_t cnt = 0;
    for (size_t e = base; cnt < G && e < M; ++cnt, e += INV_T) {
        if (cnt) fe_store_wm(pre + (size_t)(cnt - 1) * N * TT, TT, gt, run);
        fe_load_wm(x, v, M, e);
        fe_mul(run, run, x);
    }
    Fe<F> P = run, S = run;
    warp_prefix_suffix(P, S, lane);
    if (lane == 31) fe_store(s_wt + warp * N, P);
    __syncthreads();
    if (warp == 0) {
        Fe<F> w, P2, S2, inv;
        if (lane < NW)
            fe_load(w, s_wt + lane * N);
        else
            fe_one(w);
        P2 = w;
        S2 = w;
        warp_prefix_suffix(P2, S2, lane);
        Fe<F> tot;
#pragma unroll
        for (int q = 0; q < N; ++q) tot.v[q] = __shfl_sync(0xffffffffu, P2.v[q], 31);
        if (lane == 0) fe_inv(inv, tot);
#pragma unroll
        for (int q = 0; q < N; ++q) inv.v[q] = __shfl_sync(0xffffffffu, inv.v[q], 0);
        warp_exclude_self(inv, P2, S2, lane);  // 1 / (warp lane's product)
        __syncwarp();
        if (lane < NW) fe_store(s_wt + lane * N, inv);
    }
    __syncthreads();
    Fe<F> r;
    fe_load(r, s_wt + warp * N);
    warp_exclude_self(r, P, S, lane);  // 1 / run
    for (int j = (int)cnt - 1; j > 0; --j) {
        const size_t e = base + (size_t)j * INV_T;
        Fe<F> p;
        fe_load_wm(x, v, M, e);
        fe_load_wm(p, pre + (size_t)(j - 1) * N * TT, TT, gt);
        fe_mul(p, p, r);  // 1 / x_j
        fe_mul(r, r, x);
        fe_store_wm(v, M, e, p);
    }
    if (cnt) fe_store_wm(v, M, base, r);
}

// Fold level l >= 2: the level's (big bucket, group) items are flattened by
// the prefix of group counts and spread over the whole grid.  Group q of
// bucket g sums FK consecutive items of its previous level (records
// rec_first[t0+1 ..] at level 2); the level that reaches one group writes the
// bucket's total to rec_first[t0 + 1].
template <class C>
__global__ void __launch_bounds__(128) k_fold(FoldArgs a, int level, const uint32_t* __restrict__ in,
                                              uint32_t* __restrict__ out) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;
    const uint32_t base = a.prefix[0];  // the level's slice of the all-levels scan
    const uint32_t total = a.prefix[a.big_cap] - base;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += gridDim.x * blockDim.x) {
        uint32_t lo_k = 0, hi_k = a.big_cap;  // largest k with prefix[k] - base <= i
        while (hi_k - lo_k > 1) {
            const uint32_t mid = (lo_k + hi_k) >> 1;
            if (a.prefix[mid] - base <= i)
                lo_k = mid;
            else
                hi_k = mid;
        }
        const uint32_t g = a.big_list[1 + lo_k];
        const uint32_t q = i - (a.prefix[lo_k] - base);
        const uint32_t o = a.offsets[g], c = a.offsets[g + 1] - o;
        uint32_t t0, n_prev, n_cur;
        fold_sizes(o, c, a.K, a.FK, level, t0, n_prev, n_cur);
        const uint32_t lo = q * (uint32_t)a.FK, hi = min(lo + (uint32_t)a.FK, n_prev);
        Xyzz<F> acc, x;
        xyzz_load(acc, in + (size_t)(t0 + 1 + lo) * PW);
        for (uint32_t j = lo + 1; j < hi; ++j) {
            xyzz_load(x, in + (size_t)(t0 + 1 + j) * PW);
            xyzz_add(acc, x);
        }
        uint32_t* dst = (n_cur == 1) ? a.rec_first : out;
        xyzz_store(dst + (size_t)(t0 + 1 + q) * PW, acc);
    }
}

template <class F>
__device__ __forceinline__ void xyzz_dbl_n(Xyzz<F>& p, int k) {
    for (int i = 0; i < k; ++i) xyzz_dbl(p, p);
}

// R += B_g, gathering the bucket's pieces from the chunk records (see
// k_accumulate for where each piece lives).  All pieces go through one
// addition call site, so lanes whose buckets are split differently stay
// converged instead of serialising through separate inlined copies.
template <class F>
__device__ __forceinline__ void bucket_add(const SmXyzz<F, RED_THREADS>& R, const RedArgs& a, uint32_t g) {
    constexpr int PW = 4 * F::N;
    const uint32_t o = a.offsets[g], c = a.offsets[g + 1] - o;
    if (c == 0) return;
    const uint32_t t0 = o / a.K, t1 = (o + c - 1) / a.K;
    const uint32_t* first;
    uint32_t npieces;
    if (t0 == t1) {
        const uint32_t e0 = t0 * a.K, e1 = min(e0 + a.K, a.offsets[a.B]);
        first = (o == e0) ? a.rec_first + (size_t)t0 * PW
                : (o + c == e1) ? a.rec_last + (size_t)t0 * PW
                                : a.buckets + (size_t)g * PW;
        npieces = 1;
    } else {
        first = ((o == t0 * a.K) ? a.rec_first : a.rec_last) + (size_t)t0 * PW;
        // a big bucket's records t0+1..t1 were folded into rec_first[t0+1]
        npieces = 1 + ((t1 - t0 > (uint32_t)a.K2) ? 1u : (t1 - t0));
    }
    for (uint32_t k = 0; k < npieces; ++k) {
        const uint32_t* src = (k == 0) ? first : a.rec_first + (size_t)(t0 + k) * PW;
        xyzz_add(R, GXyzz<F>{src});
    }
}

// bucket_add for a quad: R is held (identically) by the quad's four lanes
// and every piece joins with the quad addition.
template <class F>
__device__ __forceinline__ void bucket_add_quad(Xyzz<F>& R, const RedArgs& a, uint32_t g) {
    constexpr int PW = 4 * F::N;
    const uint32_t o = a.offsets[g], c = a.offsets[g + 1] - o;
    if (c == 0) return;
    const uint32_t t0 = o / a.K, t1 = (o + c - 1) / a.K;
    const uint32_t* first;
    uint32_t npieces;
    if (t0 == t1) {
        const uint32_t e0 = t0 * a.K, e1 = min(e0 + a.K, a.offsets[a.B]);
        first = (o == e0) ? a.rec_first + (size_t)t0 * PW
                : (o + c == e1) ? a.rec_last + (size_t)t0 * PW
                                : a.buckets + (size_t)g * PW;
        npieces = 1;
    } else {
        first = ((o == t0 * a.K) ? a.rec_first : a.rec_last) + (size_t)t0 * PW;
        npieces = 1 + ((t1 - t0 > (uint32_t)a.K2) ? 1u : (t1 - t0));
    }
    for (uint32_t k = 0; k < npieces; ++k) {
        Xyzz<F> x;
        xyzz_load(x, (k == 0) ? first : a.rec_first + (size_t)(t0 + k) * PW);
        xyzz_add_quad(R, x);
    }
}

// Shared-memory XYZZ arrays are word-major: word i of slot t lives at
// sm[i * RED_THREADS + t], so a warp touching its 32 slots hits 32 banks.
template <class F>
__device__ __forceinline__ void sm_load(Xyzz<F>& p, const uint32_t* sm, int t) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) {
        p.X.v[i] = sm[(i)*RED_THREADS + t];
        p.Y.v[i] = sm[(F::N + i) * RED_THREADS + t];
        p.ZZ.v[i] = sm[(2 * F::N + i) * RED_THREADS + t];
        p.ZZZ.v[i] = sm[(3 * F::N + i) * RED_THREADS + t];
    }
}
template <class F>
__device__ __forceinline__ void sm_store(uint32_t* sm, int t, const Xyzz<F>& p) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) {
        sm[(i)*RED_THREADS + t] = p.X.v[i];
        sm[(F::N + i) * RED_THREADS + t] = p.Y.v[i];
        sm[(2 * F::N + i) * RED_THREADS + t] = p.ZZ.v[i];
        sm[(3 * F::N + i) * RED_THREADS + t] = p.ZZZ.v[i];
    }
}

// In-place suffix scan over the first `width` slots of sm (a power of two
// <= RED_THREADS; every thread of the block calls it):
// afterwards slot t = sum_{t' >= t} old slot t'.
template <class F>
__device__ __forceinline__ void smem_suffix_scan(uint32_t* sm, int width = RED_THREADS) {
    const int t = threadIdx.x;
    for (int d = 1; d < width; d <<= 1) {
        Xyzz<F> y, o;
        if (t < width) {
            sm_load(y, sm, t);
            if (t + d < width) {
                sm_load(o, sm, t + d);
                xyzz_add(y, o);
            }
        }
        __syncthreads();
        if (t < width) sm_store(sm, t, y);
        __syncthreads();
    }
}

// In-place tree sum over the first `width` slots of sm (a power of two <=
// RED_THREADS; every thread of the block calls it): afterwards slot 0 = sum.
template <class F>
__device__ __forceinline__ void smem_tree_sum(uint32_t* sm, int width = RED_THREADS) {
    const int t = threadIdx.x;
    for (int d = width >> 1; d >= 1; d >>= 1) {
        if (t < d) {
            Xyzz<F> y, o;
            sm_load(y, sm, t);
            sm_load(o, sm, t + d);
            xyzz_add(y, o);
            sm_store(sm, t, y);
        }
        __syncthreads();
    }
}

// The same scans over width <= RED_THREADS / 4 slots with one quad of lanes
// per slot (slot = threadIdx.x / 4) and the quad addition: a quarter of the
// depth in product latencies.  Every thread of the block calls them.
template <class F>
__device__ __forceinline__ void smem_suffix_scan_quad(uint32_t* sm, int width) {
    const int sl = threadIdx.x >> 2;
    for (int d = 1; d < width; d <<= 1) {
        Xyzz<F> y, o;
        if (sl < width) {
            sm_load(y, sm, sl);
            if (sl + d < width) {
                sm_load(o, sm, sl + d);
                xyzz_add_quad(y, o);
            }
        }
        __syncthreads();
        if (sl < width && (threadIdx.x & 3) == 0) sm_store(sm, sl, y);
        __syncthreads();
    }
}

template <class F>
__device__ __forceinline__ void smem_tree_sum_quad(uint32_t* sm, int width) {
    const int sl = threadIdx.x >> 2;
    for (int d = width >> 1; d >= 1; d >>= 1) {
        Xyzz<F> y, o;
        if (sl < d) {
            sm_load(y, sm, sl);
            sm_load(o, sm, sl + d);
            xyzz_add_quad(y, o);
        }
        __syncthreads();
        if (sl < d && (threadIdx.x & 3) == 0) sm_store(sm, sl, y);
        __syncthreads();
    }
}

// One level of a tree sum over shared-memory points (slot t += slot t + d
// for t < d; every thread of the block calls it, a barrier follows): one
// thread per slot while d > RED_QSLOTS, else one quad per slot with the
// quad addition, its scratch in slots 2d + 2t and 2d + 2t + 1 (free at this
// level of a tree over 4d or fewer live slots).
template <class F>
__device__ __forceinline__ void smem_tree_level(uint32_t* sm, int d) {
    using SP = SmXyzz<F, RED_THREADS>;
    const int me = threadIdx.x;
    if (d > RED_QSLOTS) {
        if (me < d) xyzz_add(SP{sm + me}, SP{sm + me + d});
    } else {
        const int sl = me >> 2;
        if (sl < d)
            xyzz_add_quad_sm(SP{sm + sl}, SP{sm + sl + d}, SP{sm + 2 * d + 2 * sl},
                             SP{sm + 2 * d + 2 * sl + 1});
    }
    __syncthreads();
}

// Reduction stage 2 of window w over its nb <= RED_THREADS stage-1 results
// (Fb, Sb):  V = sum_b Fb + BLK * sum_{b>=1} Y_b + Y_0, Y_b = sum_{b'>=b} Sb',
// then the window weight 2^shift.  Run by all threads of the stage-1 block
// that finished the window last (reduce_tail), in its shared memory (two
// RED_THREADS-slot point arrays); the other blocks' results are read through
// L2 (ld.global.cg), after the fence that ordered their stores before their
// completion count.
template <class C>
__device__ __forceinline__ void reduce_window(const RedArgs& a, uint32_t w, uint32_t* smr) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;
    uint32_t* sA = smr;
    uint32_t* sB = smr + RED_THREADS * PW;
    const WinDesc wd = a.wins[w];
    const uint32_t t = threadIdx.x;
    {
        Xyzz<F> Fb, Sb;
        xyzz_set_inf(Fb);
        xyzz_set_inf(Sb);
        if (t < wd.nb) {
            xyzz_load_cg(Fb, a.blk_out + ((size_t)(wd.blk_base + t) * 2) * PW);
            xyzz_load_cg(Sb, a.blk_out + ((size_t)(wd.blk_base + t) * 2 + 1) * PW);
        }
        sm_store(sA, (int)t, Sb);
        sm_store(sB, (int)t, Fb);
    }
    __syncthreads();
    // slots nb .. RED_THREADS-1 hold infinity: scan and sum only the power of
    // two that covers the window's stage-1 blocks
    int width = 1;
    while (width < (int)wd.nb) width <<= 1;
    const bool quad = width <= RED_QSLOTS;
    if (quad)
        smem_suffix_scan_quad<F>(sA, width);
    else
        smem_suffix_scan<F>(sA, width);
    Xyzz<F> Y0;
    if (t == 0) {
        sm_load(Y0, sA, 0);
        Xyzz<F> inf;
        xyzz_set_inf(inf);
        sm_store(sA, 0, inf);
    }
    __syncthreads();
    if (quad) {
        smem_tree_sum_quad<F>(sA, width);
        smem_tree_sum_quad<F>(sB, width);
    } else {
        smem_tree_sum<F>(sA, width);
        smem_tree_sum<F>(sB, width);
    }
    // Warp 0 finishes: V = [blk] (sum over b >= 1 of Y_b) + sum Fb + Y_0,
    // then the window weight 2^(c*w) by the doubling chain with its products
    // spread over the warp's lanes (two product latencies per doubling).
    if (t < 32) {
        Xyzz<F> V, u;
        sm_load(V, sA, 0);
        xyzz_mul_small_warp(V, wd.blk);
        if (t == 0) {
            sm_load(u, sB, 0);
            xyzz_add(V, u);
            xyzz_add(V, Y0);
            sm_store(sA, 0, V);
        }
        __syncwarp();
        // the doubling chain on a contiguous copy in sB (free now); an empty
        // window (the carry window of 256-bit windows is empty for scalars
        // below 2^255) skips it: it would be the longest
        uint32_t* pv = sB;
        if (t == 0) {
            sm_load(V, sA, 0);
            xyzz_store(pv, V);
        }
        __syncwarp();
        if (!SmXyzz<F, 1>{pv}.is_inf()) xyzz_dbl_chain_warp_sm<F>(pv, wd.shift, sB + PW);
        if (t == 0) SmXyzz<F, 1>{pv}.to_global(a.win_out + (size_t)w * PW);
    }
}

// V = [k] V for a small k by double-and-add on a point in shared memory (4N
// consecutive words), the doublings spread over the warp (xyzz_dbl_warp_sm),
// the additions on lane 0; tmp: 7N words, R: 4N words of shared scratch.
// All 32 lanes must call it.
template <class F>
__device__ __forceinline__ void xyzz_mul_small_warp_sm(uint32_t* p, uint32_t k, uint32_t* tmp,
                                                       uint32_t* R) {
    using S1 = SmXyzz<F, 1>;
    const int lane = threadIdx.x & 31;
    if (k == 0) {
        if (lane == 0) S1{p}.set_inf();
        __syncwarp();
        return;
    }
    if (lane == 0) xyzz_copy(S1{R}, S1{p});
    __syncwarp();
    for (int b = 30 - __clz(k); b >= 0; --b) {
        xyzz_dbl_warp_sm<F>(p, tmp);
        if ((k >> b) & 1u) {
            if (lane == 0) xyzz_add(S1{p}, S1{R});
            __syncwarp();
        }
    }
}

// reduce_window for the two-blocks-per-SM stage-1 kernel (at most 128
// registers a thread): every point stays in shared memory (SmXyzz) as in
// k_reduce_blocks, the scan and trees one slot per thread, the [blk] product
// and the doubling chain on warp 0 (xyzz_dbl_warp_sm, xyzz_dbl_chain_warp_sm).
// smr holds two RED_THREADS-slot point arrays and three stash points
// (red_blocks_smem).
template <class C>
__device__ __forceinline__ void reduce_window_sm(const RedArgs& a, uint32_t w, uint32_t* smr) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;
    using SP = SmXyzz<F, RED_THREADS>;
    using S1 = SmXyzz<F, 1>;
    uint32_t* sA = smr;
    uint32_t* sB = smr + RED_THREADS * PW;
    uint32_t* sX = smr + 2 * RED_THREADS * PW;
    const WinDesc wd = a.wins[w];
    const int me = threadIdx.x;
    int width = 1;
    while (width < (int)wd.nb) width <<= 1;
    if (me < width) {
        if (me < (int)wd.nb) {
            // Sb -> slot of sA, Fb -> slot of sB (word j at [j * RED_THREADS])
            const uint4* g =
                reinterpret_cast<const uint4*>(a.blk_out + ((size_t)(wd.blk_base + me) * 2) * PW);
#pragma unroll 4
            for (int k = 0; k < PW / 4; ++k) {
                const uint4 f = __ldcg(g + k);
                const uint4 v = __ldcg(g + PW / 4 + k);
                sB[(4 * k) * RED_THREADS + me] = f.x;
                sB[(4 * k + 1) * RED_THREADS + me] = f.y;
                sB[(4 * k + 2) * RED_THREADS + me] = f.z;
                sB[(4 * k + 3) * RED_THREADS + me] = f.w;
                sA[(4 * k) * RED_THREADS + me] = v.x;
                sA[(4 * k + 1) * RED_THREADS + me] = v.y;
                sA[(4 * k + 2) * RED_THREADS + me] = v.z;
                sA[(4 * k + 3) * RED_THREADS + me] = v.w;
            }
        } else {
            SP{sA + me}.set_inf();
            SP{sB + me}.set_inf();
        }
    }
    __syncthreads();
    // sum of Fb -> stash 0
    for (int d = width >> 1; d >= 1; d >>= 1) smem_tree_level<F>(sB, d);
    if (me == 0) xyzz_copy(S1{sX}, SP{sB});
    // suffix scan of Sb over the width slots, ping-pong between sA and sB
    uint32_t* src = sA;
    uint32_t* dst = sB;
    for (int d = 1; d < width; d <<= 1) {
        if (width > RED_QSLOTS) {
            if (me < width) {
                const SP o{dst + me};
                xyzz_copy(o, SP{src + me});
                if (me + d < width) xyzz_add(o, SP{src + me + d});
            }
        } else {
            // one quad per slot; scratch in dst slots width + 2 sl, + 1
            const int sl = me >> 2, ql = me & 3;
            if (sl < width) {
                Fe<F> c;
                SP{src + sl}.get(ql, c);
                SP{dst + sl}.put(ql, c);
                __syncwarp(0xFu << (me & 28));
                if (sl + d < width)
                    xyzz_add_quad_sm(SP{dst + sl}, SP{src + sl + d}, SP{dst + width + 2 * sl},
                                     SP{dst + width + 2 * sl + 1});
            }
        }
        __syncthreads();
        uint32_t* tmp = src;
        src = dst;
        dst = tmp;
    }
    if (me == 0) {
        xyzz_copy(S1{sX + PW}, SP{src});  // Y_0
        SP{src}.set_inf();                // the tree below sums Y_b for b >= 1
    }
    __syncthreads();
    for (int d = width >> 1; d >= 1; d >>= 1) smem_tree_level<F>(src, d);
    // Warp 0: V = [blk] (sum over b >= 1 of Y_b) + sum Fb + Y_0, then the
    // window weight 2^shift; dst is free scratch now.
    if (me < 32) {
        uint32_t* pv = dst;
        uint32_t* tmp = dst + PW;
        uint32_t* R = dst + PW + 7 * F::N;
        if (me == 0) xyzz_copy(S1{pv}, SP{src});
        __syncwarp();
        xyzz_mul_small_warp_sm<F>(pv, wd.blk, tmp, R);
        if (me == 0) {
            xyzz_add(S1{pv}, S1{sX});
            xyzz_add(S1{pv}, S1{sX + PW});
        }
        __syncwarp();
        // an empty window (the carry window of 256-bit windows is empty for
        // scalars below 2^255) skips its chain: it would be the longest
        if (!S1{pv}.is_inf()) xyzz_dbl_chain_warp_sm<F>(pv, wd.shift, tmp);
        if (me == 0) S1{pv}.to_global(a.win_out + (size_t)w * PW);
    }
}

// End of a stage-1 block: thread 0 has stored the block's (Fb, Sb).  It
// fences those stores and counts the block done for its window; the block
// that completes the window's count runs the window's stage 2 at once, so
// the windows' doubling chains (the longest first: blocks run top window
// first) overlap the remaining stage-1 blocks instead of following them.
// No block waits for another.  win_done holds one zeroed counter per window.
template <class C, bool SMEM_ONLY>
__device__ __forceinline__ void reduce_tail(const RedArgs& a, uint32_t win, uint32_t nb,
                                            uint32_t* smr) {
    __shared__ uint32_t s_last;
    __syncthreads();  // every thread is done with smr
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(a.win_done + win, 1u);
        s_last = done + 1u == nb;
        if (s_last) __threadfence();
    }
    __syncthreads();
    if (!s_last) return;
    if constexpr (SMEM_ONLY)
        reduce_window_sm<C>(a, win, smr);
    else
        reduce_window<C>(a, win, smr);
}

// Reduction stage 1 for small bucket counts (latency-bound: few blocks),
// one quad per slot, RED_QSLOTS slots of S buckets per block, the quad
// addition throughout; the same outputs as k_reduce_blocks (Fb, Sb per
// block, with blk = RED_QSLOTS * S buckets per block).
template <class C>
__global__ void __launch_bounds__(RED_THREADS) k_reduce_blocks_quad(RedArgs a) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;
    extern __shared__ __align__(16) uint32_t smr[];
    uint32_t* sA = smr;
    uint32_t* sB = smr + RED_THREADS * PW;
    const uint32_t bi = gridDim.x - 1u - blockIdx.x;  // top window first
    const BlkDesc bd = a.blks[bi];
    const WinDesc wd = a.wins[bd.win];
    const uint32_t S = wd.S;
    const int sl = threadIdx.x >> 2;
    const uint32_t first = bd.b * wd.blk + (uint32_t)sl * S;
    {
        Xyzz<F> R, T;
        xyzz_set_inf(R);
        xyzz_set_inf(T);
        for (int j = (int)S - 1; j >= 0; --j) {
            if (first + (uint32_t)j < wd.Mw) bucket_add_quad(R, a, wd.bucket_base + first + (uint32_t)j);
            if (j > 0) xyzz_add_quad(T, R);
        }
        if ((threadIdx.x & 3) == 0) {
            sm_store(sA, sl, R);
            sm_store(sB, sl, T);
        }
    }
    __syncthreads();
    smem_tree_sum_quad<F>(sB, RED_QSLOTS);    // sum of T: slot 0 of sB
    smem_suffix_scan_quad<F>(sA, RED_QSLOTS); // Y_t = sum_{t' >= t} R_t'
    Xyzz<F> Y0;
    if (threadIdx.x < 32) sm_load(Y0, sA, 0);
    __syncthreads();
    if (threadIdx.x == 0) {
        Xyzz<F> inf;
        xyzz_set_inf(inf);
        sm_store(sA, 0, inf);
    }
    __syncthreads();
    smem_tree_sum_quad<F>(sA, RED_QSLOTS);    // sum of Y_t, t >= 1
    if (threadIdx.x < 32) {
        // Fb = [S] (sum of Y_t, t >= 1) + sum of T_t; Sb = Y_0
        Xyzz<F> V, u;
        sm_load(V, sA, 0);
        xyzz_mul_small_warp(V, S);
        if (threadIdx.x == 0) {
            sm_load(u, sB, 0);
            xyzz_add(V, u);
            xyzz_store(a.blk_out + ((size_t)bi * 2) * PW, V);
            xyzz_store(a.blk_out + ((size_t)bi * 2 + 1) * PW, Y0);
        }
    }
    reduce_tail<C, false>(a, bd.win, wd.nb, smr);
}

// Reduction stage 1.  Block -> (window, b) via its BlkDesc.  Thread t owns
// S consecutive buckets of the block's range (S sized by the planner to fill
// one wave evenly); with R_t = sum_j B and T_t = sum_j j B (j relative), the
// block's
//   Fb = sum_k k B_k = sum_t T_t + S * sum_{t>=1} Y_t,   Sb = Y_0,
// where Y_t = sum_{t'>=t} R_t' (suffix scan in shared memory).
// Every point lives in shared memory (SmXyzz): sA holds R_t, sB holds T_t,
// and the two double as the ping-pong buffers of the scan once T is summed;
// sX holds three stashed points (sum of T, Y_0, a copy for the [S] product).
// Registers carry only the addition formula's temporaries, so two 256-thread
// blocks fit per SM.
template <class C>
__global__ void __launch_bounds__(RED_THREADS, 2) k_reduce_blocks(RedArgs a) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;
    using SP = SmXyzz<F, RED_THREADS>;
    using S1 = SmXyzz<F, 1>;
    extern __shared__ __align__(16) uint32_t smr[];
    uint32_t* sA = smr;
    uint32_t* sB = smr + RED_THREADS * PW;
    uint32_t* sX = smr + 2 * RED_THREADS * PW;
    const uint32_t bi = gridDim.x - 1u - blockIdx.x;  // top window first
    const BlkDesc bd = a.blks[bi];
    const WinDesc wd = a.wins[bd.win];
    const uint32_t S = wd.S;
    const uint32_t first = bd.b * wd.blk + threadIdx.x * S;
    const int me = threadIdx.x;
    {
        const SP R{sA + me}, T{sB + me};
        R.set_inf();
        T.set_inf();
        for (int j = (int)S - 1; j >= 0; --j) {
            if (first + (uint32_t)j < wd.Mw) bucket_add(R, a, wd.bucket_base + first + (uint32_t)j);
            if (j > 0) xyzz_add(T, R);
        }
    }
    __syncthreads();
    // sum of T_t -> stash 0
    for (int d = RED_THREADS >> 1; d >= 1; d >>= 1) smem_tree_level<F>(sB, d);
    if (me == 0) xyzz_copy(S1{sX}, SP{sB});
    // suffix scan of R_t, ping-pong between sA and sB (8 steps: ends in sA)
    uint32_t* src = sA;
    uint32_t* dst = sB;
    for (int d = 1; d < RED_THREADS; d <<= 1) {
        const SP o{dst + me};
        xyzz_copy(o, SP{src + me});
        if (me + d < RED_THREADS) xyzz_add(o, SP{src + me + d});
        __syncthreads();
        uint32_t* tmp = src;
        src = dst;
        dst = tmp;
    }
    if (me == 0) {
        xyzz_copy(S1{sX + PW}, SP{src});  // Y_0
        SP{src}.set_inf();                // the tree below sums Y_t for t >= 1
    }
    __syncthreads();
    for (int d = RED_THREADS >> 1; d >= 1; d >>= 1) smem_tree_level<F>(src, d);
    if (me == 0) {
        // Fb = [S] (sum of Y_t, t >= 1) + sum of T_t, by double-and-add
        const SP Fb{src};
        const S1 R{sX + 2 * PW};
        xyzz_copy(R, Fb);
        for (int b = 30 - __clz(S); b >= 0; --b) {
            xyzz_dbl(Fb);
            if ((S >> b) & 1u) xyzz_add(Fb, R);
        }
        xyzz_add(Fb, S1{sX});
        Fb.to_global(a.blk_out + ((size_t)bi * 2) * PW);
        S1{sX + PW}.to_global(a.blk_out + ((size_t)bi * 2 + 1) * PW);
    }
    reduce_tail<C, true>(a, bd.win, wd.nb, smr);
}

// Sum of each item's (already weighted) windows, then affine + wire
// (+ compressed for BLS12-381).  One warp per item: quad q (lanes 4q..4q+3)
// sums windows q, q + 8, q + 16, ... with the quad addition, then three
// shuffle levels fold the eight quads' sums into quad 0 (at 17 windows: five
// quad additions deep instead of sixteen serial additions), and lane 0
// converts and encodes.
constexpr int COMBINE_WARPS = 4;

template <class F>
__device__ __forceinline__ void xyzz_shfl_down(Xyzz<F>& r, const Xyzz<F>& p, int d) {
#pragma unroll
    for (int k = 0; k < F::N; ++k) {
        r.X.v[k] = __shfl_down_sync(0xffffffffu, p.X.v[k], d);
        r.Y.v[k] = __shfl_down_sync(0xffffffffu, p.Y.v[k], d);
        r.ZZ.v[k] = __shfl_down_sync(0xffffffffu, p.ZZ.v[k], d);
        r.ZZZ.v[k] = __shfl_down_sync(0xffffffffu, p.ZZZ.v[k], d);
    }
}

template <class C>
__global__ void __launch_bounds__(COMBINE_WARPS * 32)
    k_combine(const ItemDesc* __restrict__ items, uint32_t n_items,
              const uint32_t* __restrict__ wins, uint8_t* __restrict__ out_wire,
              uint8_t* __restrict__ out_comp) {
    using F = typename C::F;
    constexpr int PW = 4 * F::N;
    const uint32_t i = blockIdx.x * COMBINE_WARPS + (threadIdx.x >> 5);
    if (i >= n_items) return;  // whole warps
    const int lane = threadIdx.x & 31;
    const int q = lane >> 2;
    const ItemDesc it = items[i];
    Xyzz<F> acc, t;
    xyzz_set_inf(acc);
    if (it.n != 0) {
        // windows arrive already weighted by 2^(c*w): a plain sum
        for (uint32_t w = (uint32_t)q; w < it.Wr; w += 8) {
            xyzz_load(t, wins + (size_t)(it.win_base + w) * PW);
            xyzz_add_quad(acc, t);
        }
    }
    for (int d = 16; d >= 4; d >>= 1) {
        xyzz_shfl_down(t, acc, d);
        if (lane >= d) xyzz_set_inf(t);  // no partner: nothing to add
        xyzz_add_quad(acc, t);
    }
    if (lane != 0) return;
    uint8_t* ow = out_wire + (size_t)it.out_index * C::WIRE;
    uint8_t* oc = out_comp ? out_comp + (size_t)it.out_index * 48 : nullptr;
    Affine<F> af;
    const bool fin = xyzz_to_affine(af, acc);
    Fe<F> x, y;
    if (fin) {
        fe_from_mont(x, af.x);
        fe_from_mont(y, af.y);
        fe_to_be_bytes(ow, x);
        fe_to_be_bytes(ow + F::BYTES, y);
    } else {
        for (int k = 0; k < C::WIRE; ++k) ow[k] = 0;
    }
    if (oc && C::CURVE_ID == 2) {
        // ZCash/IETF compressed form: bit7 compressed, bit6 infinity,
        // bit5 iff y > (p-1)/2, i.e. 2y > p.
        if (!fin) {
            oc[0] = 0xC0;
            for (int k = 1; k < 48; ++k) oc[k] = 0;
        } else {
            uint32_t y2[F::N];
            uint32_t cy = 0;
            for (int k = 0; k < F::N; ++k) {
                y2[k] = (y.v[k] << 1) | cy;
                cy = y.v[k] >> 31;
            }
            // 2y > p  <=>  p - 2y borrows (2y != p since p is odd)
            int64_t bw = 0;
            for (int k = 0; k < F::N; ++k) {
                const int64_t v = (int64_t)F::P(k) - (int64_t)y2[k] - bw;
                bw = v < 0 ? 1 : 0;
            }
            for (int k = 0; k < 48; ++k) oc[k] = ow[k];
            oc[0] |= 0x80;
            if (bw) oc[0] |= 0x20;
        }
    }
}

template <class C>
struct MsmLaunchImpl {
    using F = typename C::F;
    static void wire_to_table(const uint8_t* w, uint32_t* t, size_t n, size_t glv_stride,
                              cudaStream_t st) {
        if (!n) return;
        if (((uintptr_t)w & 15) == 0)
            k_wire_to_table<C, true><<<ceil_div_u(n, 128), 128, 0, st>>>(w, t, n, glv_stride);
        else
            k_wire_to_table<C, false><<<ceil_div_u(n, 128), 128, 0, st>>>(w, t, n, glv_stride);
        KB_LAUNCH_CHECK();
    }
    static void table_to_wire(const uint32_t* t, uint8_t* w, size_t n, cudaStream_t st) {
        if (!n) return;
        k_table_to_wire<C><<<ceil_div_u(n, 128), 128, 0, st>>>(t, w, n);
        KB_LAUNCH_CHECK();
    }
    static void recode(const ItemDesc* items, uint32_t n_items, unsigned long long first,
                       unsigned long long count, const uint32_t* scalars, const uint32_t* table,
                       uint32_t* keys, uint32_t* vals, cudaStream_t st) {
        if (!count) return;
        k_recode<C><<<ceil_div_u(count, 256), 256, 0, st>>>(items, n_items, first, count, scalars,
                                                           table, keys, vals);
        KB_LAUNCH_CHECK();
    }
    // One pairing level over T0 = ceil(slots / PAIR_J) threads; scratch holds
    // pair_scratch_words(T0, N) words.
    static void pair_level(const PairArgs& a, uint32_t T0, uint32_t* scratch, cudaStream_t st) {
        if (!T0) return;
        constexpr int N = F::N;
        uint32_t* pre0 = scratch;
        uint32_t* tot = pre0 + (size_t)(PAIR_J - 1) * N * T0;
        k_pair_fwd<C><<<ceil_div_u(T0, 256), 256, 0, st>>>(a, T0, pre0, tot);
        KB_LAUNCH_CHECK();
        const InvGeom g = inv_geom(T0);
        k_inv_wide<F><<<g.nb, INV_T, 0, st>>>(tot, T0, g.G, tot + (size_t)N * T0);
        KB_LAUNCH_CHECK();
        if (a.dst_off)
            k_pair_bwd<C, true><<<ceil_div_u(T0, 256), 256, 0, st>>>(a, T0, pre0, tot);
        else
            k_pair_bwd<C, false><<<ceil_div_u(T0, 256), 256, 0, st>>>(a, T0, pre0, tot);
        KB_LAUNCH_CHECK();
    }
    static void accumulate(const AccArgs& a, unsigned grid, cudaStream_t st) {
        k_accumulate<C><<<grid, 128, 0, st>>>(a);
        KB_LAUNCH_CHECK();
    }
    static void fold(const FoldArgs& a, int level, const uint32_t* in, uint32_t* out,
                     unsigned grid, cudaStream_t st) {
        k_fold<C><<<grid, 128, 0, st>>>(a, level, in, out);
        KB_LAUNCH_CHECK();
    }
    static size_t red_smem() { return (size_t)2 * RED_THREADS * 4 * F::N * 4; }
    static size_t red_blocks_smem() { return red_smem() + (size_t)3 * 4 * F::N * 4; }
    static void reduce_blocks(const RedArgs& a, unsigned nblk, cudaStream_t st) {
        if (!nblk) return;
        set_smem_attr((const void*)k_reduce_blocks<C>, red_blocks_smem());
        k_reduce_blocks<C><<<nblk, RED_THREADS, red_blocks_smem(), st>>>(a);
        KB_LAUNCH_CHECK();
    }
    static void reduce_blocks_quad(const RedArgs& a, unsigned nblk, cudaStream_t st) {
        if (!nblk) return;
        set_smem_attr((const void*)k_reduce_blocks_quad<C>, red_smem());
        k_reduce_blocks_quad<C><<<nblk, RED_THREADS, red_smem(), st>>>(a);
        KB_LAUNCH_CHECK();
    }
    static void combine(const ItemDesc* items, uint32_t n_items, const uint32_t* wins,
                        uint8_t* ow, uint8_t* oc, cudaStream_t st) {
        if (!n_items) return;
        k_combine<C><<<ceil_div_u(n_items, COMBINE_WARPS), COMBINE_WARPS * 32, 0, st>>>(
            items, n_items, wins, ow, oc);
        KB_LAUNCH_CHECK();
    }
    static int accumulate_occupancy() {
        int blocks = 0;
        KB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_accumulate<C>, 128, 0));
        return blocks;
    }
    static MsmLaunchers table() {
        MsmLaunchers L;
        L.wire_to_table = &wire_to_table;
        L.table_to_wire = &table_to_wire;
        L.recode = &recode;
        L.accumulate = &accumulate;
        L.pair_level = &pair_level;
        L.fold = &fold;
        L.reduce_blocks = &reduce_blocks;
        L.reduce_blocks_quad = &reduce_blocks_quad;
        L.combine = &combine;
        L.accumulate_occupancy = &accumulate_occupancy;
        L.point_words = 4 * F::N;
        L.table_words = 2 * F::N;
        L.wire_bytes = C::WIRE;
        return L;
    }
};

}  // namespace kb200
