// Montgomery field arithmetic on 32-bit limbs for sm_100a.
//
// Four prime fields, all with R = 2^(32N) (the same Montgomery domain as the
// reference's 64-bit-limb code, so Montgomery images are bit-identical):
//   FpBLS : BLS12-381 base field, N = 12   (bls/cpp/bls12_381_fp.hpp:83-98)
//   FrBLS : BLS12-381 scalar field, N = 8  (kzg/cpp/kzg_oracle.hpp:66-90)
//   FpBN  : BN254 base field, N = 8        (bn254/cpp/bn254_fp.hpp:75-89)
//   FrBN  : BN254 scalar field, N = 8      (bn254/cpp/bn254_fp.hpp:79-97)
//
// Multiplication (fe_mul_inl): a one-level Karatsuba double-width product
// followed by a word-serial Montgomery reduction; every partial-product row
// is two carry chains -- the even-indexed products (lo into t[j], hi into
// t[j+1]) and then the odd-indexed ones -- written as consecutive
// mad.lo.cc / madc.hi.cc instructions.  Every value is kept fully reduced in
// [0, p); all four moduli satisfy 2p < 2^(32N).
#pragma once
#include <cstdint>

#define KB_DEV __device__ __forceinline__
#define KB_HD __host__ __device__ __forceinline__

namespace kb200 {

// ---------------------------------------------------------------------------
// PTX carry-chain primitives.  volatile keeps the compiler from moving them
// relative to one another, so a chain written as consecutive calls stays a
// chain on the condition-code register.
// ---------------------------------------------------------------------------
KB_DEV uint32_t mad_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
KB_DEV uint32_t madc_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
KB_DEV uint32_t madc_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
KB_DEV uint32_t addc_u32(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("addc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
KB_DEV uint32_t add_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
KB_DEV uint32_t addc_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
KB_DEV uint32_t sub_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
KB_DEV uint32_t subc_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
KB_DEV uint32_t subc_u32(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

// ---------------------------------------------------------------------------
// Field parameters.  Limbs are little-endian 32-bit words.
// ---------------------------------------------------------------------------
struct FpBLS {
    static constexpr int N = 12;
    static constexpr int BYTES = 48;
    static constexpr uint32_t M0 = 0xfffcfffdu;  // -p^-1 mod 2^32
    KB_HD static constexpr uint32_t P(int i) {
        constexpr uint32_t t[12] = {0xffffaaab, 0xb9feffff, 0xb153ffff, 0x1eabfffe,
                                    0xf6b0f624, 0x6730d2a0, 0xf38512bf, 0x64774b84,
                                    0x434bacd7, 0x4b1ba7b6, 0x397fe69a, 0x1a0111ea};
        return t[i];
    }
    KB_HD static constexpr uint32_t R1(int i) {
        constexpr uint32_t t[12] = {0x0002fffd, 0x76090000, 0xc40c0002, 0xebf4000b,
                                    0x53c758ba, 0x5f489857, 0x70525745, 0x77ce5853,
                                    0xa256ec6d, 0x5c071a97, 0xfa80e493, 0x15f65ec3};
        return t[i];
    }
    KB_HD static constexpr uint32_t R2(int i) {
        constexpr uint32_t t[12] = {0x1c341746, 0xf4df1f34, 0x09d104f1, 0x0a76e6a6,
                                    0x4c95b6d5, 0x8de5476c, 0x939d83c0, 0x67eb88a9,
                                    0xb519952d, 0x9a793e85, 0x92cae3aa, 0x11988fe5};
        return t[i];
    }
};

struct FrBLS {
    static constexpr int N = 8;
    static constexpr int BYTES = 32;
    static constexpr uint32_t M0 = 0xffffffffu;
    KB_HD static constexpr uint32_t P(int i) {
        constexpr uint32_t t[8] = {0x00000001, 0xffffffff, 0xfffe5bfe, 0x53bda402,
                                   0x09a1d805, 0x3339d808, 0x299d7d48, 0x73eda753};
        return t[i];
    }
    KB_HD static constexpr uint32_t R1(int i) {
        constexpr uint32_t t[8] = {0xfffffffe, 0x00000001, 0x00034802, 0x5884b7fa,
                                   0xecbc4ff5, 0x998c4fef, 0xacc5056f, 0x1824b159};
        return t[i];
    }
    KB_HD static constexpr uint32_t R2(int i) {
        constexpr uint32_t t[8] = {0xf3f29c6d, 0xc999e990, 0x87925c23, 0x2b6cedcb,
                                   0x7254398f, 0x05d31496, 0x9f59ff11, 0x0748d9d9};
        return t[i];
    }
};

struct FpBN {
    static constexpr int N = 8;
    static constexpr int BYTES = 32;
    static constexpr uint32_t M0 = 0xe4866389u;
    KB_HD static constexpr uint32_t P(int i) {
        constexpr uint32_t t[8] = {0xd87cfd47, 0x3c208c16, 0x6871ca8d, 0x97816a91,
                                   0x8181585d, 0xb85045b6, 0xe131a029, 0x30644e72};
        return t[i];
    }
    KB_HD static constexpr uint32_t R1(int i) {
        constexpr uint32_t t[8] = {0xc58f0d9d, 0xd35d438d, 0xf5c70b3d, 0x0a78eb28,
                                   0x7879462c, 0x666ea36f, 0x9a07df2f, 0x0e0a77c1};
        return t[i];
    }
    KB_HD static constexpr uint32_t R2(int i) {
        constexpr uint32_t t[8] = {0x538afa89, 0xf32cfc5b, 0xd44501fb, 0xb5e71911,
                                   0x0a417ff6, 0x47ab1eff, 0xcab8351f, 0x06d89f71};
        return t[i];
    }
};

struct FrBN {
    static constexpr int N = 8;
    static constexpr int BYTES = 32;
    static constexpr uint32_t M0 = 0xefffffffu;
    KB_HD static constexpr uint32_t P(int i) {
        constexpr uint32_t t[8] = {0xf0000001, 0x43e1f593, 0x79b97091, 0x2833e848,
                                   0x8181585d, 0xb85045b6, 0xe131a029, 0x30644e72};
        return t[i];
    }
    KB_HD static constexpr uint32_t R1(int i) {
        constexpr uint32_t t[8] = {0x4ffffffb, 0xac96341c, 0x9f60cd29, 0x36fc7695,
                                   0x7879462e, 0x666ea36f, 0x9a07df2f, 0x0e0a77c1};
        return t[i];
    }
    KB_HD static constexpr uint32_t R2(int i) {
        constexpr uint32_t t[8] = {0xae216da7, 0x1bb8e645, 0xe35c59e3, 0x53fe3ab1,
                                   0x53bb8085, 0x8c49833d, 0x7f4e44a5, 0x0216d0b1};
        return t[i];
    }
};

// ---------------------------------------------------------------------------
// Element type and arithmetic.
// ---------------------------------------------------------------------------
template <class F>
struct Fe {
    uint32_t v[F::N];
};

template <class F>
KB_DEV void fe_zero(Fe<F>& a) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) a.v[i] = 0;
}
template <class F>
KB_DEV void fe_one(Fe<F>& a) {  // 1 in Montgomery form (R mod p)
#pragma unroll
    for (int i = 0; i < F::N; ++i) a.v[i] = F::R1(i);
}
template <class F>
KB_DEV bool fe_is_zero(const Fe<F>& a) {
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < F::N; ++i) acc |= a.v[i];
    return acc == 0;
}
template <class F>
KB_DEV bool fe_eq(const Fe<F>& a, const Fe<F>& b) {
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < F::N; ++i) acc |= a.v[i] ^ b.v[i];
    return acc == 0;
}

// t[0..H] += a[0..H) * b for a word b (an (H+1)-word window whose sum the
// caller guarantees fits): the even-indexed partial products as one carry
// chain, then the odd-indexed ones as another.
template <int H>
KB_DEV void mac_row(uint32_t* t, const uint32_t* a, uint32_t b) {
    t[0] = mad_lo_cc(a[0], b, t[0]);
    t[1] = madc_hi_cc(a[0], b, t[1]);
#pragma unroll
    for (int j = 2; j < H; j += 2) {
        t[j] = madc_lo_cc(a[j], b, t[j]);
        t[j + 1] = madc_hi_cc(a[j], b, t[j + 1]);
    }
    t[H] = addc_u32(t[H], 0);
    t[1] = mad_lo_cc(a[1], b, t[1]);
    t[2] = madc_hi_cc(a[1], b, t[2]);
#pragma unroll
    for (int j = 3; j < H; j += 2) {
        t[j] = madc_lo_cc(a[j], b, t[j]);
        t[j + 1] = madc_hi_cc(a[j], b, t[j + 1]);
    }
}

// r[0..2H) = a * b for H-word a, b (schoolbook rows).
template <int H>
KB_DEV void mul_words(uint32_t* r, const uint32_t* a, const uint32_t* b) {
#pragma unroll
    for (int i = 0; i < 2 * H; ++i) r[i] = 0;
#pragma unroll
    for (int i = 0; i < H; ++i) mac_row<H>(r + i, a, b[i]);
}

// r = t - p if t >= p else t (t < 2p, N words).
template <class F>
KB_DEV void reduce_once(Fe<F>& r, const uint32_t* t) {
    constexpr int N = F::N;
    uint32_t d[N];
    d[0] = sub_cc(t[0], F::P(0));
#pragma unroll
    for (int i = 1; i < N; ++i) d[i] = subc_cc(t[i], F::P(i));
    uint32_t borrow = subc_u32(0, 0);  // 0xffffffff if t < p
#pragma unroll
    for (int i = 0; i < N; ++i) r.v[i] = borrow ? t[i] : d[i];
}

template <class F>
KB_DEV void mont_reduce_wide(Fe<F>& r, uint32_t* T);

// r = a * b * R^-1 mod p, inputs and output in [0, p).
//
// The double-width product T = a * b uses one level of Karatsuba on the
// N/2-word halves: a_lo b_lo and a_hi b_hi, and (a_lo + a_hi)(b_lo + b_hi)
// minus both (the halves' sums carry one extra bit each, added back as
// masked words), 3 (N/2)^2 word products instead of N^2.  The Montgomery
// reduction then runs word by word over T (separated operand scanning): row
// i adds m_i p at word i with m_i = T[i] * (-p^-1 mod 2^32), as two carry
// chains whose final carries are kept aside and added to the upper half at
// the end, so no carry has to ripple through T row by row.  The result is
// (T + m p) / 2^(32N) < 2p, then one conditional subtraction.  Integer
// multiply-adds: 6N^2/4 + 2N^2 + N against 4N^2 + 3N for the interleaved
// (CIOS) form, e.g. 516 against 612 for N = 12; measured on a B200 at
// saturation, 29.4 against 27.1 G products/s (BLS12-381 Fp) and 62.1
// against 58.3 (BN254 Fp).
template <class F>
KB_DEV void fe_mul_ks_inl(Fe<F>& r, const Fe<F>& a, const Fe<F>& b) {
    constexpr int N = F::N, H = N / 2;
    static_assert(N % 4 == 0, "halves of an even number of words");
    uint32_t T[2 * N];
    mul_words<H>(T, a.v, b.v);
    mul_words<H>(T + N, a.v + H, b.v + H);
    uint32_t sa[H], sb[H];
    sa[0] = add_cc(a.v[0], a.v[H]);
#pragma unroll
    for (int k = 1; k < H; ++k) sa[k] = addc_cc(a.v[k], a.v[H + k]);
    const uint32_t ca = addc_u32(0, 0);
    sb[0] = add_cc(b.v[0], b.v[H]);
#pragma unroll
    for (int k = 1; k < H; ++k) sb[k] = addc_cc(b.v[k], b.v[H + k]);
    const uint32_t cb = addc_u32(0, 0);
    // M = (sa + ca 2^(32H)) (sb + cb 2^(32H)) - a_lo b_lo - a_hi b_hi, N + 1 words
    uint32_t M[N + 1];
    mul_words<H>(M, sa, sb);
    M[N] = 0;
    const uint32_t mca = 0u - ca, mcb = 0u - cb;
    M[H] = add_cc(M[H], sb[0] & mca);
#pragma unroll
    for (int k = 1; k < H; ++k) M[H + k] = addc_cc(M[H + k], sb[k] & mca);
    M[N] = addc_u32(M[N], 0);
    M[H] = add_cc(M[H], sa[0] & mcb);
#pragma unroll
    for (int k = 1; k < H; ++k) M[H + k] = addc_cc(M[H + k], sa[k] & mcb);
    M[N] = addc_u32(M[N], ca & cb);
    M[0] = sub_cc(M[0], T[0]);
#pragma unroll
    for (int k = 1; k < N; ++k) M[k] = subc_cc(M[k], T[k]);
    M[N] = subc_u32(M[N], 0);
    M[0] = sub_cc(M[0], T[N]);
#pragma unroll
    for (int k = 1; k < N; ++k) M[k] = subc_cc(M[k], T[N + k]);
    M[N] = subc_u32(M[N], 0);
    T[H] = add_cc(T[H], M[0]);
#pragma unroll
    for (int k = 1; k <= N; ++k) T[H + k] = addc_cc(T[H + k], M[k]);
#pragma unroll
    for (int k = H + N + 1; k < 2 * N; ++k) T[k] = addc_cc(T[k], 0);
    mont_reduce_wide<F>(r, T);
}

// r = T * 2^(-32N) mod p for a double-width T < p 2^(32N) (2N words, T is
// consumed): word-serial Montgomery reduction; row i adds m_i p at word i,
// m_i = T[i] (-p^-1 mod 2^32), as two carry chains whose final carries pc
// are kept aside and added to the upper half at the end, so no carry has to
// ripple through T row by row.  (T + m p) / 2^(32N) < 2p, then one
// conditional subtraction.
template <class F>
KB_DEV void mont_reduce_wide(Fe<F>& r, uint32_t* T) {
    constexpr int N = F::N;
    // reduction rows; pc[k] collects the chains' carries into word N + k
    uint32_t pc[N + 1];
#pragma unroll
    for (int k = 0; k <= N; ++k) pc[k] = 0;
    // A modulus with low words 1 and 2^32 - 1 (the BLS12-381 scalar field r)
    // needs no multiply for them: m_i = -T[i] (as -p^-1 = 2^32 - 1), m_i * 1
    // = m_i makes word i zero with a carry iff T[i] != 0, and m_i (2^32 - 1)
    // = (T[i], T[i] ? ~T[i] : 0) as (low, high) words.  Five integer
    // multiply-adds fewer per row, 40 of 232 per product for N = 8.
    constexpr bool LOW_ONE = F::P(0) == 1u && F::P(1) == 0xffffffffu;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const uint32_t t = T[i];
        const uint32_t m = LOW_ONE ? 0u - t : t * F::M0;
        if constexpr (LOW_ONE) {
            T[i] = add_cc(t, m);
            T[i + 1] = addc_cc(T[i + 1], 0u);
        } else {
            T[i] = mad_lo_cc(m, F::P(0), T[i]);
            T[i + 1] = madc_hi_cc(m, F::P(0), T[i + 1]);
        }
#pragma unroll
        for (int j = 2; j < N; j += 2) {
            T[i + j] = madc_lo_cc(m, F::P(j), T[i + j]);
            T[i + j + 1] = madc_hi_cc(m, F::P(j), T[i + j + 1]);
        }
        pc[i] = addc_u32(pc[i], 0);
        if constexpr (LOW_ONE) {
            const uint32_t hi = t ? ~t : 0u;
            T[i + 1] = add_cc(T[i + 1], t);
            T[i + 2] = addc_cc(T[i + 2], hi);
        } else {
            T[i + 1] = mad_lo_cc(m, F::P(1), T[i + 1]);
            T[i + 2] = madc_hi_cc(m, F::P(1), T[i + 2]);
        }
#pragma unroll
        for (int j = 3; j < N - 1; j += 2) {
            T[i + j] = madc_lo_cc(m, F::P(j), T[i + j]);
            T[i + j + 1] = madc_hi_cc(m, F::P(j), T[i + j + 1]);
        }
        T[i + N - 1] = madc_lo_cc(m, F::P(N - 1), T[i + N - 1]);
        T[i + N] = madc_hi_cc(m, F::P(N - 1), T[i + N]);
        pc[i + 1] = addc_u32(pc[i + 1], 0);
    }
    // (T + m p) / 2^(32N) = T[N..2N) + pc, below 2p < 2^(32N)
    uint32_t U[N];
    U[0] = add_cc(T[N], pc[0]);
#pragma unroll
    for (int k = 1; k < N; ++k) U[k] = addc_cc(T[N + k], pc[k]);
    reduce_once<F>(r, U);
}


// r = a * b * R^-1 mod p in the interleaved (CIOS) form: for each word b_i,
// the row a b_i and the reduction row m p (m = t_0 (-p^-1) mod 2^32) are
// added into an (N+1)-word accumulator, 4N^2 + 3N integer multiply-adds.
// It keeps far fewer values live than fe_mul_ks_inl (the accumulator instead
// of the double-width product), so kernels that inline several products at
// one place use it; the out-of-line fe_mul uses the Karatsuba form.  Measured
// on the BLS12-381 MSM at 2^22: every product in the Karatsuba form but the
// two inlined recovery products of the pairing levels 27.19 ms; those two
// in the Karatsuba form too 27.11 ms (more registers); all in this form
// 28.21 ms; the two recovery products out of line 28.03 ms.  With the later
// kernels (tiled ranking, fused reduction) the Karatsuba recovery products
// lost on both curves: pair stage 20.35 -> 20.61 ms (BLS12-381 2^22), 39.57
// -> 39.70 ms (BN254 2^24), with BLS12-381 spills of 260 bytes.
template <class F>
KB_DEV void fe_mul_inl(Fe<F>& r, const Fe<F>& a, const Fe<F>& b) {
    constexpr int N = F::N;
    uint32_t p[N];
#pragma unroll
    for (int i = 0; i < N; ++i) p[i] = F::P(i);
    uint32_t t[N + 1];
#pragma unroll
    for (int i = 0; i <= N; ++i) t[i] = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        mac_row<N>(t, a.v, b.v[i]);
        uint32_t m = t[0] * F::M0;
        mac_row<N>(t, p, m);
#pragma unroll
        for (int j = 0; j < N; ++j) t[j] = t[j + 1];
        t[N] = 0;
    }
    reduce_once<F>(r, t);
}

// Out-of-line copy: one instance of the ~640-instruction product per
// kernel instead of one per call site, which keeps large kernels (bucket
// reduction, window combine) inside the instruction cache.
template <class F>
__device__ __noinline__ Fe<F> fe_mul_call(Fe<F> a, Fe<F> b) {
    Fe<F> r;
    fe_mul_ks_inl<F>(r, a, b);
    return r;
}

#ifndef KB_MUL_INLINE
#define KB_MUL_INLINE 0
#endif

template <class F>
KB_DEV void fe_mul(Fe<F>& r, const Fe<F>& a, const Fe<F>& b) {
#if KB_MUL_INLINE
    fe_mul_inl<F>(r, a, b);
#else
    r = fe_mul_call<F>(a, b);
#endif
}

template <class F>
KB_DEV void fe_sqr(Fe<F>& r, const Fe<F>& a) {
    fe_mul<F>(r, a, a);
}
template <class F>
KB_DEV void fe_sqr_inl(Fe<F>& r, const Fe<F>& a) {
    fe_mul_inl<F>(r, a, a);
}

template <class F>
KB_DEV void fe_add(Fe<F>& r, const Fe<F>& a, const Fe<F>& b) {
    constexpr int N = F::N;
    uint32_t s[N];
    s[0] = add_cc(a.v[0], b.v[0]);
#pragma unroll
    for (int i = 1; i < N; ++i) s[i] = addc_cc(a.v[i], b.v[i]);
    reduce_once<F>(r, s);
}

template <class F>
KB_DEV void fe_sub(Fe<F>& r, const Fe<F>& a, const Fe<F>& b) {
    constexpr int N = F::N;
    uint32_t d[N];
    d[0] = sub_cc(a.v[0], b.v[0]);
#pragma unroll
    for (int i = 1; i < N; ++i) d[i] = subc_cc(a.v[i], b.v[i]);
    uint32_t mask = subc_u32(0, 0);
    r.v[0] = add_cc(d[0], F::P(0) & mask);
#pragma unroll
    for (int i = 1; i < N; ++i) r.v[i] = addc_cc(d[i], F::P(i) & mask);
}

template <class F>
KB_DEV void fe_neg(Fe<F>& r, const Fe<F>& a) {
    Fe<F> z;
    fe_zero(z);
    fe_sub<F>(r, z, a);
}

template <class F>
KB_DEV void fe_dbl(Fe<F>& r, const Fe<F>& a) {
    fe_add<F>(r, a, a);
}

// Conversions between canonical and Montgomery form.  to_mont accepts any
// N-word value (it need not be below p): the CIOS bound keeps the product
// below 2p because R^2 mod p < p, so the result is the canonical image of
// (a mod p) -- the same reduction the reference's to_mont performs.
template <class F>
KB_DEV void fe_to_mont(Fe<F>& r, const Fe<F>& a) {
    Fe<F> r2;
#pragma unroll
    for (int i = 0; i < F::N; ++i) r2.v[i] = F::R2(i);
    fe_mul<F>(r, a, r2);
}
template <class F>
KB_DEV void fe_from_mont(Fe<F>& r, const Fe<F>& a) {
    Fe<F> one;
    fe_zero(one);
    one.v[0] = 1;
    fe_mul<F>(r, a, one);
}

// Exponent word i of p - 2, with the borrow propagated (BLS12-381 r has
// low word 1, so p - 2 borrows from word 1 there).
template <class F>
KB_HD constexpr uint32_t pm2_word(int i) {
    uint32_t borrow = 2;
    uint32_t w = 0;
    for (int k = 0; k <= i; ++k) {
        const uint32_t pk = F::P(k);
        w = pk - borrow;
        borrow = pk < borrow ? 1u : 0u;
    }
    return w;
}

// a^(p-2) by left-to-right square-and-multiply with 4-bit fixed windows:
// the reference the binary-GCD inversion is checked against on the device
// (kb200_field_inverse_check).
template <class F>
__device__ __noinline__ void fe_inv_fermat(Fe<F>& r, const Fe<F>& a) {
    Fe<F> tab[16];
    fe_one(tab[0]);
    tab[1] = a;
#pragma unroll 1
    for (int i = 2; i < 16; ++i) fe_mul<F>(tab[i], tab[i - 1], a);
    Fe<F> acc;
    fe_one(acc);
    bool started = false;
#pragma unroll 1
    for (int w = F::N * 8 - 1; w >= 0; --w) {
        const uint32_t word = pm2_word<F>(w >> 3);
        const uint32_t nib = (word >> ((w & 7) * 4)) & 15u;
        if (started) {
#pragma unroll 1
            for (int s = 0; s < 4; ++s) fe_sqr<F>(acc, acc);
        }
        if (nib) {
            if (started) {
                fe_mul<F>(acc, acc, tab[nib]);
            } else {
                acc = tab[nib];
                started = true;
            }
        }
    }
    r = acc;
}

// ---- Inversion by the optimized binary GCD ---------------------------------
// Pornin, "Optimized Binary GCD for Modular Inversion" (IACR ePrint 2020/972),
// Algorithm 2 with 32-bit words: each outer step runs 31 divsteps on 64-bit
// approximations of (a, b) (their low 31 bits and top 33 bits), collecting
// the 2x2 update (f0, g0; f1, g1) with |f| + |g| <= 2^31, then applies it to
// the full values: a <- (a f0 + b g0) / 2^31, b <- (a f1 + b g1) / 2^31 (exact
// divisions; a negative result is negated with its row of factors).  The
// companions u, v follow with the same factors and a Montgomery division by
// 2^31, so a = u y and b = v y (mod p) hold throughout; starting from u =
// R^2 the final v is (aR)^-1 R^2 = a^-1 R, the Montgomery form of the inverse.
// ceil((2 len(p) - 1) / 31) outer steps always end with b = 1 for y != 0.
// Fixed trip counts and a branch-free divstep: the lanes of a warp stay
// converged, so it serves bulk conversions as well as single results.
namespace gcd_detail {

template <class F>
KB_HD constexpr int bit_length_p() {
    int top = F::N - 1;
    while (top > 0 && F::P(top) == 0) --top;
    uint32_t w = F::P(top);
    int b = 0;
    while (w) {
        ++b;
        w >>= 1;
    }
    return 32 * top + b;
}

// r (N + 2 words, two's complement) = x f + y g for non-negative N-word x, y
// and |f|, |g| <= 2^31.
template <int N>
KB_DEV void lin_comb(uint32_t (&r)[N + 2], const uint32_t (&x)[N], const uint32_t (&y)[N], int64_t f,
                     int64_t g) {
    const uint32_t fa = (uint32_t)(f < 0 ? -f : f), ga = (uint32_t)(g < 0 ? -g : g);
    const uint32_t mx = f < 0 ? 0xffffffffu : 0u, my = g < 0 ? 0xffffffffu : 0u;
    uint64_t cx = 0, cy = 0, c = (uint64_t)(mx & 1u) + (my & 1u);
#pragma unroll
    for (int i = 0; i <= N; ++i) {
        uint32_t px, py;
        if (i < N) {
            const uint64_t tx = (uint64_t)x[i] * fa + cx;
            const uint64_t ty = (uint64_t)y[i] * ga + cy;
            px = (uint32_t)tx;
            py = (uint32_t)ty;
            cx = tx >> 32;
            cy = ty >> 32;
        } else {
            px = (uint32_t)cx;
            py = (uint32_t)cy;
        }
        const uint64_t s = (uint64_t)(px ^ mx) + (py ^ my) + c;
        r[i] = (uint32_t)s;
        c = s >> 32;
    }
    r[N + 1] = mx + my + (uint32_t)c;
}

// r (N + 1 words, two's complement) = t / 2^31 for a two's-complement t of
// N + 2 words whose low 31 bits are zero.
template <int N>
KB_DEV void shr31(uint32_t (&r)[N + 1], const uint32_t (&t)[N + 2]) {
#pragma unroll
    for (int i = 0; i <= N; ++i) r[i] = (t[i] >> 31) | (t[i + 1] << 1);
}

// x (N + 1 words, two's complement) -> |x| in place; returns true if x < 0.
template <int N>
KB_DEV bool abs_in_place(uint32_t (&x)[N + 1]) {
    const bool neg = (x[N] >> 31) != 0;
    const uint32_t m = neg ? 0xffffffffu : 0u;
    uint64_t c = neg ? 1u : 0u;
#pragma unroll
    for (int i = 0; i <= N; ++i) {
        const uint64_t s = (uint64_t)(x[i] ^ m) + c;
        x[i] = (uint32_t)s;
        c = s >> 32;
    }
    return neg;
}

// (u f + v g) / 2^31 mod p for u, v in [0, p): the sum plus q p with
// q = -sum p^-1 mod 2^31 divides exactly; the quotient lies in (-2p, 2p).
template <class F>
KB_DEV void mont_comb(uint32_t (&r)[F::N], const uint32_t (&u)[F::N], const uint32_t (&v)[F::N], int64_t f,
                      int64_t g) {
    constexpr int N = F::N;
    uint32_t t[N + 2];
    lin_comb<N>(t, u, v, f, g);
    const uint32_t q = (t[0] * F::M0) & 0x7fffffffu;
    uint64_t c = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const uint64_t s = (uint64_t)F::P(i) * q + t[i] + c;
        t[i] = (uint32_t)s;
        c = s >> 32;
    }
    {
        const uint64_t s = (uint64_t)t[N] + c;
        t[N] = (uint32_t)s;
        t[N + 1] += (uint32_t)(s >> 32);
    }
    uint32_t w[N + 1];
    shr31<N>(w, t);
    // into [0, p): add p while negative (at most twice), subtract p once if >= p
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const uint32_t m = (w[N] >> 31) ? 0xffffffffu : 0u;
        uint64_t cc = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const uint64_t s = (uint64_t)w[i] + (F::P(i) & m) + cc;
            w[i] = (uint32_t)s;
            cc = s >> 32;
        }
        w[N] += (uint32_t)cc;
    }
    uint32_t d[N];
    int64_t br = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const int64_t s = (int64_t)w[i] - F::P(i) + br;
        d[i] = (uint32_t)s;
        br = s >> 32;
    }
    const bool ge = (int64_t)w[N] + br >= 0;
#pragma unroll
    for (int i = 0; i < N; ++i) r[i] = ge ? d[i] : w[i];
}

// Bits [s, s + 33) of the N-word x, for 31 <= s <= 32 N - 33.
template <int N>
KB_DEV uint64_t top33(const uint32_t (&x)[N], int s) {
    const int wi = s >> 5, sh = s & 31;
    uint32_t w0 = 0, w1 = 0, w2 = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        w0 = k == wi ? x[k] : w0;
        w1 = k == wi + 1 ? x[k] : w1;
        w2 = k == wi + 2 ? x[k] : w2;
    }
    uint64_t v = (((uint64_t)w1 << 32) | w0) >> sh;
    if (sh) v |= (uint64_t)w2 << (64 - sh);
    return v & ((1ull << 33) - 1);
}

}  // namespace gcd_detail

template <class F>
__device__ __noinline__ void fe_inv_gcd(Fe<F>& r, const Fe<F>& y) {
    using namespace gcd_detail;
    constexpr int N = F::N;
    constexpr int STEPS = (2 * bit_length_p<F>() - 1 + 30) / 31;
    uint32_t a[N], b[N], u[N], v[N];
    uint32_t any = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        a[i] = y.v[i];
        b[i] = F::P(i);
        u[i] = F::R2(i);
        v[i] = 0;
        any |= y.v[i];
    }
#pragma unroll 1
    for (int it = 0; it < STEPS; ++it) {
        // n = max(len a, len b, 64); approximations from the low 31 and top 33 bits
        int n = 64;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const uint32_t w = a[k] | b[k];
            n = w ? max(n, 32 * k + 32 - __clz(w)) : n;
        }
        uint64_t ab = (a[0] & 0x7fffffffu) | (top33<N>(a, n - 33) << 31);
        uint64_t bb = (b[0] & 0x7fffffffu) | (top33<N>(b, n - 33) << 31);
        int64_t f0 = 1, g0 = 0, f1 = 0, g1 = 1;
#pragma unroll 1
        for (int j = 0; j < 31; ++j) {
            const bool odd = (ab & 1) != 0;
            const bool sw = odd && ab < bb;
            const uint64_t a2 = sw ? bb : ab, b2 = sw ? ab : bb;
            const int64_t nf0 = sw ? f1 : f0, ng0 = sw ? g1 : g0;
            const int64_t nf1 = sw ? f0 : f1, ng1 = sw ? g0 : g1;
            ab = odd ? a2 - b2 : a2;
            bb = b2;
            f0 = odd ? nf0 - nf1 : nf0;
            g0 = odd ? ng0 - ng1 : ng0;
            f1 = nf1;
            g1 = ng1;
            ab >>= 1;
            f1 <<= 1;
            g1 <<= 1;
        }
        uint32_t ta[N + 2], tb[N + 2], na[N + 1], nb[N + 1];
        lin_comb<N>(ta, a, b, f0, g0);
        lin_comb<N>(tb, a, b, f1, g1);
        shr31<N>(na, ta);
        shr31<N>(nb, tb);
        if (abs_in_place<N>(na)) {
            f0 = -f0;
            g0 = -g0;
        }
        if (abs_in_place<N>(nb)) {
            f1 = -f1;
            g1 = -g1;
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            a[i] = na[i];
            b[i] = nb[i];
        }
        uint32_t nu[N], nv[N];
        mont_comb<F>(nu, u, v, f0, g0);
        mont_comb<F>(nv, u, v, f1, g1);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            u[i] = nu[i];
            v[i] = nv[i];
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) r.v[i] = any ? v[i] : 0u;
}

// 1/a in Montgomery form (0 for 0).
template <class F>
KB_DEV void fe_inv(Fe<F>& r, const Fe<F>& a) {
    fe_inv_gcd<F>(r, a);
}

// Load / store helpers for canonical little-endian words.
template <class F>
KB_DEV void fe_load(Fe<F>& r, const uint32_t* src) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) r.v[i] = src[i];
}
template <class F>
KB_DEV void fe_store(uint32_t* dst, const Fe<F>& a) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) dst[i] = a.v[i];
}

// The same through 16-byte accesses: src / dst 16-byte aligned (point
// records are 2N or 4N words and N is a multiple of 4).
template <class F>
KB_DEV void fe_load16(Fe<F>& r, const uint32_t* src) {
    static_assert(F::N % 4 == 0, "16-byte field access needs N % 4 == 0");
    const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
    for (int k = 0; k < F::N / 4; ++k) {
        const uint4 v = s[k];
        r.v[4 * k] = v.x;
        r.v[4 * k + 1] = v.y;
        r.v[4 * k + 2] = v.z;
        r.v[4 * k + 3] = v.w;
    }
}
template <class F>
KB_DEV void fe_store16(uint32_t* dst, const Fe<F>& a) {
    static_assert(F::N % 4 == 0, "16-byte field access needs N % 4 == 0");
    uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int k = 0; k < F::N / 4; ++k)
        d[k] = make_uint4(a.v[4 * k], a.v[4 * k + 1], a.v[4 * k + 2], a.v[4 * k + 3]);
}

// Big-endian byte string (F::BYTES long) -> little-endian words.
template <class F>
KB_DEV void fe_from_be_bytes(Fe<F>& r, const uint8_t* b) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) {
        const uint8_t* q = b + F::BYTES - 4 * (i + 1);
        r.v[i] = ((uint32_t)q[0] << 24) | ((uint32_t)q[1] << 16) | ((uint32_t)q[2] << 8) |
                 (uint32_t)q[3];
    }
}
template <class F>
KB_DEV void fe_to_be_bytes(uint8_t* b, const Fe<F>& a) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) {
        uint8_t* q = b + F::BYTES - 4 * (i + 1);
        q[0] = (uint8_t)(a.v[i] >> 24);
        q[1] = (uint8_t)(a.v[i] >> 16);
        q[2] = (uint8_t)(a.v[i] >> 8);
        q[3] = (uint8_t)a.v[i];
    }
}

}  // namespace kb200
