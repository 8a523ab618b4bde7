/*
 * Word-prime NTT oracle (TEST INFRASTRUCTURE ONLY): a plain-C restatement of
 * the reference's ntt_forward / ntt_inverse (ntt/c-abi/c_ntt.cpp:81-179) and
 * the three bodies they dispatch to:
 *
 *   n <= 2^16, modulus = 998244353 and the pinned root
 *       -> Montgomery (R = 2^32) radix-2 path, ntt/cpp/ntt.cpp:100-172
 *   n <= 2^16, any other (modulus, root)
 *       -> 128-bit-mulmod radix-2 path, ntt/cpp/ntt.cpp:176-219
 *   2^16 < n <= 2^20
 *       -> six-step path with transposed output, ntt/cpp/ntt_large.cpp:145-248
 *
 * Every path keeps the reference's arithmetic step for step (which operand is
 * reduced where, which additions check for 64-bit overflow), so outputs match
 * for every input, canonical or not.  Only the tests and the benchmark's CPU
 * leg call this file.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* Cyclone-FFT prime and its pinned 2^16-th root (ntt/cpp/ntt.hpp:43-57). */
#define CYC_Q 998244353ULL
#define CYC_ROOT 629671588ULL
#define CYC_MAX_LOG 16
#define LARGE_MAX_LOG 20
/* Montgomery constants for R = 2^32 (ntt/cpp/ntt.hpp:59-64). */
#define CYC_R_MOD_Q 301989884ULL
#define CYC_R2_MOD_Q 932051910ULL
#define CYC_QINV32 998244351ULL

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1;
    b %= q;
    while (e) {
        if (e & 1) r = mulmod(r, b, q);
        b = mulmod(b, b, q);
        e >>= 1;
    }
    return r;
}

/* --- Cyclone path arithmetic (ntt/cpp/ntt.cpp:33-66): 64-bit wrapping. --- */
static uint64_t cyc_redc(uint64_t t) {
    uint64_t m = ((t & 0xffffffffULL) * CYC_QINV32) & 0xffffffffULL;
    uint64_t u = (t + m * CYC_Q) >> 32;
    return u >= CYC_Q ? u - CYC_Q : u;
}
static uint64_t cyc_mul(uint64_t a, uint64_t b_mont) { return cyc_redc(a * b_mont); }
static uint64_t cyc_add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return s >= CYC_Q ? s - CYC_Q : s;
}
static uint64_t cyc_sub(uint64_t a, uint64_t b) { return a >= b ? a - b : a + CYC_Q - b; }

static unsigned log2_exact(size_t n) {
    unsigned l = 0;
    while (((size_t)1 << l) < n) ++l;
    return l;
}
static uint32_t bitrev(uint32_t x, unsigned bits) {
    uint32_t r = 0;
    for (unsigned i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}
/* in-place bit reversal of the elements a[0], a[s], a[2s], ... */
static void bitrev_permute(uint64_t* a, uint32_t n, unsigned logn, size_t stride) {
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t j = bitrev(i, logn);
        if (i < j) {
            uint64_t t = a[i * stride];
            a[i * stride] = a[j * stride];
            a[j * stride] = t;
        }
    }
}

static void cyclone_dit(uint64_t* a, uint32_t n, unsigned logn, int inverse) {
    bitrev_permute(a, n, logn, 1);
    for (unsigned s = 1; s <= logn; ++s) {
        const uint32_t m = 1u << s, half = m >> 1;
        uint64_t wm = powmod(CYC_ROOT, 1ULL << (CYC_MAX_LOG - s), CYC_Q);
        if (inverse) wm = powmod(wm, CYC_Q - 2, CYC_Q);
        const uint64_t wm_m = cyc_redc(wm * CYC_R2_MOD_Q);
        for (uint32_t k = 0; k < n; k += m) {
            uint64_t w = CYC_R_MOD_Q;
            for (uint32_t j = 0; j < half; ++j) {
                const uint64_t u = a[k + j];
                const uint64_t t = cyc_mul(a[k + j + half], w);
                a[k + j] = cyc_add(u, t);
                a[k + j + half] = cyc_sub(u, t);
                w = cyc_redc(w * wm_m);
            }
        }
    }
    if (inverse) {
        const uint64_t ninv_m = cyc_redc(powmod(n, CYC_Q - 2, CYC_Q) * CYC_R2_MOD_Q);
        for (uint32_t i = 0; i < n; ++i) a[i] = cyc_mul(a[i], ninv_m);
    }
}

/* --- generic small path (ntt/cpp/ntt.cpp:176-219): inputs reduced at every
 * use; the addition has no 64-bit overflow check. --- */
static void generic_dit(uint64_t* a, uint32_t n, unsigned logn, uint64_t q, uint64_t w0) {
    bitrev_permute(a, n, logn, 1);
    for (unsigned s = 1; s <= logn; ++s) {
        const uint32_t m = 1u << s, half = m >> 1;
        const uint64_t wm = powmod(w0, n / m, q);
        for (uint32_t k = 0; k < n; k += m) {
            uint64_t w = 1;
            for (uint32_t j = 0; j < half; ++j) {
                const uint64_t u = a[k + j] % q;
                const uint64_t t = mulmod(w, a[k + j + half] % q, q);
                uint64_t sum = u + t;
                if (sum >= q) sum -= q;
                a[k + j] = sum;
                a[k + j + half] = u >= t ? u - t : u + q - t;
                w = mulmod(w, wm, q);
            }
        }
    }
}

/* --- large path (ntt/cpp/ntt_large.cpp): overflow-checked addition, the
 * upper operand reduced by the product only. --- */
static uint64_t lg_add(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    if (s >= q || s < a) s -= q;
    return s;
}
static void large_sub_ntt(uint64_t* a, uint32_t n, unsigned logn, size_t stride,
                          uint64_t w_n, uint64_t q) {
    bitrev_permute(a, n, logn, stride);
    for (unsigned s = 1; s <= logn; ++s) {
        const uint32_t m = 1u << s, half = m >> 1;
        const uint64_t wm = powmod(w_n, (uint64_t)n >> s, q);
        for (uint32_t k = 0; k < n; k += m) {
            uint64_t w = 1;
            for (uint32_t j = 0; j < half; ++j) {
                const size_t lo = (size_t)(k + j) * stride, hi = lo + (size_t)half * stride;
                const uint64_t u = a[lo];
                const uint64_t t = mulmod(w, a[hi], q);
                a[lo] = lg_add(u, t, q);
                a[hi] = u >= t ? u - t : u + q - t;
                w = mulmod(w, wm, q);
            }
        }
    }
}

static void diag_multiply(uint64_t* a, uint32_t n1, uint32_t n2, uint64_t w, uint64_t q) {
    for (uint32_t i = 0; i < n1; ++i) {
        const uint64_t base = powmod(w, i, q);
        uint64_t cur = 1;
        for (uint32_t j = 0; j < n2; ++j) {
            a[(size_t)i * n2 + j] = mulmod(a[(size_t)i * n2 + j], cur, q);
            cur = mulmod(cur, base, q);
        }
    }
}

static void large_transform(uint64_t* a, uint32_t n, uint64_t q, uint64_t omega_2n, int inverse) {
    const unsigned logn = log2_exact(n), l1 = logn / 2, l2 = logn - l1;
    const uint32_t n1 = 1u << l1, n2 = 1u << l2;
    const uint64_t wn = mulmod(omega_2n, omega_2n, q);
    const uint64_t wn_inv = powmod(wn, q - 2, q);
    const uint64_t w = inverse ? wn_inv : wn;
    const uint64_t w1 = powmod(w, n2, q), w2 = powmod(w, n1, q);
    if (!inverse) {
        for (uint32_t j = 0; j < n2; ++j) large_sub_ntt(a + j, n1, l1, n2, w1, q);
        diag_multiply(a, n1, n2, w, q);
        for (uint32_t i = 0; i < n1; ++i) large_sub_ntt(a + (size_t)i * n2, n2, l2, 1, w2, q);
    } else {
        for (uint32_t i = 0; i < n1; ++i) large_sub_ntt(a + (size_t)i * n2, n2, l2, 1, w2, q);
        diag_multiply(a, n1, n2, w, q);
        for (uint32_t j = 0; j < n2; ++j) large_sub_ntt(a + j, n1, l1, n2, w1, q);
        const uint64_t ninv = powmod(n, q - 2, q);
        for (uint32_t k = 0; k < n; ++k) a[k] = mulmod(a[k], ninv, q);
    }
}

/* Status codes of c-abi/crypto.h:60-66. */
#define ORC_OK 0
#define ORC_ERR_INPUT (-1)

static int is_pow2(size_t n) { return n != 0 && (n & (n - 1)) == 0; }

int orc_word_ntt_forward(uint64_t* a, size_t n, uint64_t q, uint64_t root) {
    if (!a || !is_pow2(n)) return ORC_ERR_INPUT;
    if (n <= ((size_t)1 << CYC_MAX_LOG)) {
        if (q == 0) return ORC_ERR_INPUT;
        if (n <= 1) return ORC_OK;
        if (q == CYC_Q && root == CYC_ROOT)
            cyclone_dit(a, (uint32_t)n, log2_exact(n), 0);
        else
            generic_dit(a, (uint32_t)n, log2_exact(n), q, root);
        return ORC_OK;
    }
    if (n > ((size_t)1 << LARGE_MAX_LOG)) return ORC_ERR_INPUT;
    if (q == 0) return ORC_ERR_INPUT; /* 2^64 needs an inverse of the even n */
    large_transform(a, (uint32_t)n, q, root, 0);
    return ORC_OK;
}

int orc_word_ntt_inverse(uint64_t* a, size_t n, uint64_t q, uint64_t root_inv) {
    if (!a || !is_pow2(n)) return ORC_ERR_INPUT;
    if (n <= ((size_t)1 << CYC_MAX_LOG)) {
        if (q == 0) return ORC_ERR_INPUT;
        if (n <= 1) return ORC_OK;
        if (q == CYC_Q && (root_inv == CYC_ROOT || root_inv == powmod(CYC_ROOT, CYC_Q - 2, CYC_Q))) {
            cyclone_dit(a, (uint32_t)n, log2_exact(n), 1);
            return ORC_OK;
        }
        generic_dit(a, (uint32_t)n, log2_exact(n), q, root_inv);
        const uint64_t ninv = powmod(n, q - 2, q);
        for (size_t i = 0; i < n; ++i) a[i] = mulmod(a[i], ninv, q);
        return ORC_OK;
    }
    if (n > ((size_t)1 << LARGE_MAX_LOG)) return ORC_ERR_INPUT;
    if (q == 0) return ORC_ERR_INPUT;
    large_transform(a, (uint32_t)n, q, powmod(root_inv, q - 2, q), 1);
    return ORC_OK;
}
