/*
 * CPU oracle (TEST INFRASTRUCTURE ONLY) -- plain-C restatement of the
 * reference's CPU path.  Never linked by the product library.
 *
 * Field arithmetic restates the reference's 64-bit-limb CIOS Montgomery code:
 *   BLS12-381 Fp : bls/cpp/bls12_381_fp.hpp:83-245
 *   BLS12-381 Fr : kzg/cpp/kzg_oracle.hpp:64-210
 *   BN254 Fp, Fr : bn254/cpp/bn254_fp.hpp:75-263
 * Group law (Jacobian, a = 0) restates add-2007-bl / dbl-2009-l as written in
 *   bls/cpp/bls12_381_g1.hpp:57-151 and bn254/cpp/bn254_g1.hpp:51-170.
 * Pippenger restates gpukit/cpp/cpu_reference/multi_pippenger.cpp:67-181.
 * The NTT restates the radix-2 DIT order of ntt/cpp/ntt.cpp:128-172 over Fr.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef uint64_t u64;

/* ------------------------------------------------------------------------ */
/* Generic Montgomery field over up to 6 64-bit limbs.                      */
/* ------------------------------------------------------------------------ */

typedef struct { u64 l[6]; } fe;

typedef struct {
    int n;          /* 64-bit limbs */
    int bytes;      /* canonical byte width at the boundary */
    fe p, r1, r2;   /* modulus, R mod p, R^2 mod p */
    u64 pinv;       /* -p^-1 mod 2^64 */
} field;

/* bls/cpp/bls12_381_fp.hpp:83-98 */
static const field F_BLS_FP = {6, 48,
    {{0xB9FEFFFFFFFFAAABULL, 0x1EABFFFEB153FFFFULL, 0x6730D2A0F6B0F624ULL,
      0x64774B84F38512BFULL, 0x4B1BA7B6434BACD7ULL, 0x1A0111EA397FE69AULL}},
    {{0x760900000002FFFDULL, 0xEBF4000BC40C0002ULL, 0x5F48985753C758BAULL,
      0x77CE585370525745ULL, 0x5C071A97A256EC6DULL, 0x15F65EC3FA80E493ULL}},
    {{0xF4DF1F341C341746ULL, 0x0A76E6A609D104F1ULL, 0x8DE5476C4C95B6D5ULL,
      0x67EB88A9939D83C0ULL, 0x9A793E85B519952DULL, 0x11988FE592CAE3AAULL}},
    0x89F3FFFCFFFCFFFDULL};
/* kzg/cpp/kzg_oracle.hpp:66-90 */
static const field F_BLS_FR = {4, 32,
    {{0xFFFFFFFF00000001ULL, 0x53BDA402FFFE5BFEULL, 0x3339D80809A1D805ULL,
      0x73EDA753299D7D48ULL}},
    {{0x00000001FFFFFFFEULL, 0x5884B7FA00034802ULL, 0x998C4FEFECBC4FF5ULL,
      0x1824B159ACC5056FULL}},
    {{0xC999E990F3F29C6DULL, 0x2B6CEDCB87925C23ULL, 0x05D314967254398FULL,
      0x0748D9D99F59FF11ULL}},
    0xFFFFFFFEFFFFFFFFULL};
/* bn254/cpp/bn254_fp.hpp:75-89 */
static const field F_BN_FP = {4, 32,
    {{0x3C208C16D87CFD47ULL, 0x97816A916871CA8DULL, 0xB85045B68181585DULL,
      0x30644E72E131A029ULL}},
    {{0xD35D438DC58F0D9DULL, 0x0A78EB28F5C70B3DULL, 0x666EA36F7879462CULL,
      0x0E0A77C19A07DF2FULL}},
    {{0xF32CFC5B538AFA89ULL, 0xB5E71911D44501FBULL, 0x47AB1EFF0A417FF6ULL,
      0x06D89F71CAB8351FULL}},
    0x87D20782E4866389ULL};
/* bn254/cpp/bn254_fp.hpp:79-97 */
static const field F_BN_FR = {4, 32,
    {{0x43E1F593F0000001ULL, 0x2833E84879B97091ULL, 0xB85045B68181585DULL,
      0x30644E72E131A029ULL}},
    {{0xAC96341C4FFFFFFBULL, 0x36FC76959F60CD29ULL, 0x666EA36F7879462EULL,
      0x0E0A77C19A07DF2FULL}},
    {{0x1BB8E645AE216DA7ULL, 0x53FE3AB1E35C59E3ULL, 0x8C49833D53BB8085ULL,
      0x0216D0B17F4E44A5ULL}},
    0xC2E1F593EFFFFFFFULL};

static const field* field_by_id(int which) {
    switch (which) {
        case 0: return &F_BLS_FP;
        case 1: return &F_BLS_FR;
        case 2: return &F_BN_FP;
        case 3: return &F_BN_FR;
        default: return NULL;
    }
}

static int fe_cmp(const field* F, const fe* a, const fe* b) {
    for (int i = F->n - 1; i >= 0; --i) {
        if (a->l[i] < b->l[i]) return -1;
        if (a->l[i] > b->l[i]) return 1;
    }
    return 0;
}
static int fe_is_zero(const field* F, const fe* a) {
    u64 acc = 0;
    for (int i = 0; i < F->n; ++i) acc |= a->l[i];
    return acc == 0;
}
static u64 raw_add(const field* F, fe* r, const fe* a, const fe* b) {
    u64 c = 0;
    for (int i = 0; i < F->n; ++i) {
        u128 t = (u128)a->l[i] + b->l[i] + c;
        r->l[i] = (u64)t;
        c = (u64)(t >> 64);
    }
    return c;
}
static u64 raw_sub(const field* F, fe* r, const fe* a, const fe* b) {
    u64 bw = 0;
    for (int i = 0; i < F->n; ++i) {
        u128 t = (u128)a->l[i] - b->l[i] - bw;
        r->l[i] = (u64)t;
        bw = (u64)(t >> 64) & 1;
    }
    return bw;
}
/* mod_add / mod_sub / neg: bls12_381_fp.hpp:129-147, :204-208 */
static fe f_add(const field* F, fe a, fe b) {
    fe t;
    u64 c = raw_add(F, &t, &a, &b);
    if (c || fe_cmp(F, &t, &F->p) >= 0) raw_sub(F, &t, &t, &F->p);
    return t;
}
static fe f_sub(const field* F, fe a, fe b) {
    fe t;
    if (raw_sub(F, &t, &a, &b)) raw_add(F, &t, &t, &F->p);
    return t;
}
static fe f_neg(const field* F, fe a) {
    if (fe_is_zero(F, &a)) return a;
    fe t;
    raw_sub(F, &t, &F->p, &a);
    return t;
}
/* CIOS Montgomery product a*b*R^-1: bls12_381_fp.hpp:153-189 (n = 6) and
 * bn254_fp.hpp:155-191 (n = 4) share this shape. */
static fe f_mul(const field* F, fe a, fe b) {
    const int n = F->n;
    u64 t[8] = {0};
    for (int i = 0; i < n; ++i) {
        u64 carry = 0;
        for (int j = 0; j < n; ++j) {
            u128 prod = (u128)a.l[j] * b.l[i] + t[j] + carry;
            t[j] = (u64)prod;
            carry = (u64)(prod >> 64);
        }
        u128 sum = (u128)t[n] + carry;
        t[n] = (u64)sum;
        t[n + 1] += (u64)(sum >> 64);
        u64 u = t[0] * F->pinv;
        carry = 0;
        for (int j = 0; j < n; ++j) {
            u128 prod = (u128)u * F->p.l[j] + t[j] + carry;
            t[j] = (u64)prod;
            carry = (u64)(prod >> 64);
        }
        sum = (u128)t[n] + carry;
        t[n] = (u64)sum;
        t[n + 1] += (u64)(sum >> 64);
        for (int j = 0; j < n + 1; ++j) t[j] = t[j + 1];
        t[n + 1] = 0;
    }
    fe r;
    memset(&r, 0, sizeof r);
    for (int i = 0; i < n; ++i) r.l[i] = t[i];
    if (t[n] != 0 || fe_cmp(F, &r, &F->p) >= 0) raw_sub(F, &r, &r, &F->p);
    return r;
}
static fe f_sqr(const field* F, fe a) { return f_mul(F, a, a); }
static fe f_to_mont(const field* F, fe a) { return f_mul(F, a, F->r2); }
static fe f_from_mont(const field* F, fe a) {
    fe one;
    memset(&one, 0, sizeof one);
    one.l[0] = 1;
    return f_mul(F, a, one);
}
static fe f_one(const field* F) { return F->r1; }
/* square-and-multiply, bls12_381_fp.hpp:220-232 */
static fe f_pow(const field* F, fe a_mont, const fe* e) {
    fe result = f_one(F), base = a_mont;
    for (int limb = 0; limb < F->n; ++limb) {
        u64 w = e->l[limb];
        for (int bit = 0; bit < 64; ++bit) {
            if ((w >> bit) & 1) result = f_mul(F, result, base);
            base = f_sqr(F, base);
        }
    }
    return result;
}
static fe f_inv(const field* F, fe a_mont) {
    fe e = F->p, two;
    memset(&two, 0, sizeof two);
    two.l[0] = 2;
    raw_sub(F, &e, &e, &two);
    return f_pow(F, a_mont, &e);
}
static fe f_from_small(const field* F, u64 v) {
    fe a;
    memset(&a, 0, sizeof a);
    a.l[0] = v;
    return f_to_mont(F, a);
}

static fe fe_from_le(const field* F, const uint8_t* b) {
    fe r;
    memset(&r, 0, sizeof r);
    for (int i = 0; i < F->bytes; ++i) r.l[i / 8] |= (u64)b[i] << (8 * (i % 8));
    return r;
}
static void fe_to_le(const field* F, const fe* a, uint8_t* b) {
    for (int i = 0; i < F->bytes; ++i) b[i] = (uint8_t)(a->l[i / 8] >> (8 * (i % 8)));
}
static fe fe_from_be(const field* F, const uint8_t* b) {
    fe r;
    memset(&r, 0, sizeof r);
    for (int i = 0; i < F->bytes; ++i) {
        int k = F->bytes - 1 - i;
        r.l[k / 8] |= (u64)b[i] << (8 * (k % 8));
    }
    return r;
}
static void fe_to_be(const field* F, const fe* a, uint8_t* b) {
    for (int i = 0; i < F->bytes; ++i) {
        int k = F->bytes - 1 - i;
        b[i] = (uint8_t)(a->l[k / 8] >> (8 * (k % 8)));
    }
}

int orc_field_mul(int which, const uint8_t* a, const uint8_t* b, uint8_t* out) {
    const field* F = field_by_id(which);
    if (!F) return -1;
    fe x = f_to_mont(F, fe_from_le(F, a)), y = f_to_mont(F, fe_from_le(F, b));
    fe z = f_from_mont(F, f_mul(F, x, y));
    fe_to_le(F, &z, out);
    return 0;
}
int orc_field_inv(int which, const uint8_t* a, uint8_t* out) {
    const field* F = field_by_id(which);
    if (!F) return -1;
    fe z = f_from_mont(F, f_inv(F, f_to_mont(F, fe_from_le(F, a))));
    fe_to_le(F, &z, out);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* G1, Jacobian coordinates, a = 0.                                        */
/* ------------------------------------------------------------------------ */

typedef struct { fe X, Y, Z; int inf; } jac;

typedef struct {
    const field* F;
    u64 b;             /* curve constant */
    int pt_bytes;      /* wire bytes per affine point */
    uint8_t gx[48], gy[48];
} curve;

static curve C_BLS, C_BN;
static int curves_ready = 0;

static void init_curves(void) {
    if (curves_ready) return;
    /* bls/cpp/bls12_381_g1.hpp:204-224 */
    static const uint8_t gx[48] = {
        0x17, 0xF1, 0xD3, 0xA7, 0x31, 0x97, 0xD7, 0x94, 0x26, 0x95, 0x63, 0x8C,
        0x4F, 0xA9, 0xAC, 0x0F, 0xC3, 0x68, 0x8C, 0x4F, 0x97, 0x74, 0xB9, 0x05,
        0xA1, 0x4E, 0x3A, 0x3F, 0x17, 0x1B, 0xAC, 0x58, 0x6C, 0x55, 0xE8, 0x3F,
        0xF9, 0x7A, 0x1A, 0xEF, 0xFB, 0x3A, 0xF0, 0x0A, 0xDB, 0x22, 0xC6, 0xBB};
    static const uint8_t gy[48] = {
        0x08, 0xB3, 0xF4, 0x81, 0xE3, 0xAA, 0xA0, 0xF1, 0xA0, 0x9E, 0x30, 0xED,
        0x74, 0x1D, 0x8A, 0xE4, 0xFC, 0xF5, 0xE0, 0x95, 0xD5, 0xD0, 0x0A, 0xF6,
        0x00, 0xDB, 0x18, 0xCB, 0x2C, 0x04, 0xB3, 0xED, 0xD0, 0x3C, 0xC7, 0x44,
        0xA2, 0x88, 0x8A, 0xE4, 0x0C, 0xAA, 0x23, 0x29, 0x46, 0xC5, 0xE7, 0xE1};
    C_BLS.F = &F_BLS_FP;
    C_BLS.b = 4;
    C_BLS.pt_bytes = 96;
    memcpy(C_BLS.gx, gx, 48);
    memcpy(C_BLS.gy, gy, 48);
    /* BN254 G1 generator (1, 2), EIP-196. */
    C_BN.F = &F_BN_FP;
    C_BN.b = 3;
    C_BN.pt_bytes = 64;
    memset(C_BN.gx, 0, 48);
    memset(C_BN.gy, 0, 48);
    C_BN.gx[31] = 1;
    C_BN.gy[31] = 2;
    curves_ready = 1;
}

static const curve* curve_by_id(uint32_t id) {
    init_curves();
    if (id == ORC_CURVE_BLS12_381) return &C_BLS;
    if (id == ORC_CURVE_BN254) return &C_BN;
    return NULL;
}

static jac jac_zero(void) {
    jac r;
    memset(&r, 0, sizeof r);
    r.inf = 1;
    return r;
}

/* dbl-2009-l: bls12_381_g1.hpp:75-110 */
static jac jac_double(const curve* C, jac p) {
    const field* F = C->F;
    if (p.inf) return p;
    if (fe_is_zero(F, &p.Y)) return jac_zero();
    fe A = f_sqr(F, p.X), B = f_sqr(F, p.Y), Cc = f_sqr(F, B);
    fe D = f_sub(F, f_sqr(F, f_add(F, p.X, B)), A);
    D = f_sub(F, D, Cc);
    D = f_add(F, D, D);
    fe E = f_add(F, f_add(F, A, A), A);
    fe Fq = f_sqr(F, E);
    fe X3 = f_sub(F, Fq, f_add(F, D, D));
    fe C8 = f_add(F, Cc, Cc);
    C8 = f_add(F, C8, C8);
    C8 = f_add(F, C8, C8);
    fe Y3 = f_sub(F, f_mul(F, E, f_sub(F, D, X3)), C8);
    fe Z3 = f_mul(F, p.Y, p.Z);
    Z3 = f_add(F, Z3, Z3);
    jac r = {X3, Y3, Z3, 0};
    return r;
}

/* add-2007-bl: bls12_381_g1.hpp:113-151 */
static jac jac_add(const curve* C, jac a, jac b) {
    const field* F = C->F;
    if (a.inf) return b;
    if (b.inf) return a;
    fe Z1Z1 = f_sqr(F, a.Z), Z2Z2 = f_sqr(F, b.Z);
    fe U1 = f_mul(F, a.X, Z2Z2), U2 = f_mul(F, b.X, Z1Z1);
    fe S1 = f_mul(F, f_mul(F, a.Y, b.Z), Z2Z2);
    fe S2 = f_mul(F, f_mul(F, b.Y, a.Z), Z1Z1);
    fe H = f_sub(F, U2, U1);
    if (fe_is_zero(F, &H)) {
        if (fe_cmp(F, &S1, &S2) == 0) return jac_double(C, a);
        return jac_zero();
    }
    fe I = f_sqr(F, f_add(F, H, H));
    fe J = f_mul(F, H, I);
    fe r_ = f_sub(F, S2, S1);
    r_ = f_add(F, r_, r_);
    fe V = f_mul(F, U1, I);
    fe X3 = f_sub(F, f_sub(F, f_sqr(F, r_), J), f_add(F, V, V));
    fe Y3 = f_sub(F, f_mul(F, r_, f_sub(F, V, X3)), f_mul(F, f_add(F, S1, S1), J));
    fe Z3 = f_sub(F, f_sub(F, f_sqr(F, f_add(F, a.Z, b.Z)), Z1Z1), Z2Z2);
    Z3 = f_mul(F, Z3, H);
    jac out = {X3, Y3, Z3, 0};
    return out;
}

static jac jac_neg(const curve* C, jac p) {
    if (p.inf) return p;
    p.Y = f_neg(C->F, p.Y);
    return p;
}

/* read_affine: gpukit/curve_traits/bls12_381_g1_first_party_traits.h:58-69 */
static jac read_point(const curve* C, const uint8_t* xy) {
    const field* F = C->F;
    int any = 0;
    for (int i = 0; i < C->pt_bytes; ++i) any |= xy[i];
    if (!any) return jac_zero();
    jac r;
    r.X = f_to_mont(F, fe_from_be(F, xy));
    r.Y = f_to_mont(F, fe_from_be(F, xy + F->bytes));
    r.Z = f_one(F);
    r.inf = 0;
    return r;
}

/* write_affine + g1_to_affine: traits .h:71-83, bls12_381_g1.hpp:57-72 */
static void write_point(const curve* C, jac p, uint8_t* xy) {
    const field* F = C->F;
    if (p.inf || fe_is_zero(F, &p.Z)) {
        memset(xy, 0, (size_t)C->pt_bytes);
        return;
    }
    fe zi = f_inv(F, p.Z), zi2 = f_sqr(F, zi), zi3 = f_mul(F, zi2, zi);
    fe x = f_from_mont(F, f_mul(F, p.X, zi2));
    fe y = f_from_mont(F, f_mul(F, p.Y, zi3));
    fe_to_be(F, &x, xy);
    fe_to_be(F, &y, xy + F->bytes);
}

/* Left-to-right double-and-add over 256 bits (variable time; test use only). */
static jac jac_mul(const curve* C, jac p, const uint8_t* k_le) {
    jac acc = jac_zero();
    for (int i = 255; i >= 0; --i) {
        acc = jac_double(C, acc);
        if ((k_le[i >> 3] >> (i & 7)) & 1) acc = jac_add(C, acc, p);
    }
    return acc;
}

static jac generator(const curve* C) {
    uint8_t g[96];
    memcpy(g, C->gx, (size_t)C->F->bytes);
    memcpy(g + C->F->bytes, C->gy, (size_t)C->F->bytes);
    return read_point(C, g);
}

int orc_g1_mul_gen(uint32_t curve_id, const uint8_t* k_le, uint8_t* result) {
    const curve* C = curve_by_id(curve_id);
    if (!C || !k_le || !result) return -1;
    write_point(C, jac_mul(C, generator(C), k_le), result);
    return 0;
}

int orc_g1_mul(uint32_t curve_id, const uint8_t* point, const uint8_t* k_le,
               uint8_t* result) {
    const curve* C = curve_by_id(curve_id);
    if (!C || !point || !k_le || !result) return -1;
    write_point(C, jac_mul(C, read_point(C, point), k_le), result);
    return 0;
}

int orc_g1_add(uint32_t curve_id, const uint8_t* p, const uint8_t* q, uint8_t* result) {
    const curve* C = curve_by_id(curve_id);
    if (!C || !p || !q || !result) return -1;
    write_point(C, jac_add(C, read_point(C, p), read_point(C, q)), result);
    return 0;
}

/* g1_is_on_curve: bls12_381_g1.hpp:195-201 */
int orc_g1_on_curve(uint32_t curve_id, const uint8_t* p) {
    const curve* C = curve_by_id(curve_id);
    if (!C || !p) return -1;
    const field* F = C->F;
    int any = 0;
    for (int i = 0; i < C->pt_bytes; ++i) any |= p[i];
    if (!any) return 1;
    fe x = fe_from_be(F, p), y = fe_from_be(F, p + F->bytes);
    if (fe_cmp(F, &x, &F->p) >= 0 || fe_cmp(F, &y, &F->p) >= 0) return 0;
    x = f_to_mont(F, x);
    y = f_to_mont(F, y);
    fe lhs = f_sqr(F, y);
    fe rhs = f_add(F, f_mul(F, f_sqr(F, x), x), f_from_small(F, C->b));
    return fe_cmp(F, &lhs, &rhs) == 0;
}

/* ------------------------------------------------------------------------ */
/* Pippenger: gpukit/cpp/cpu_reference/multi_pippenger.cpp:67-181          */
/* ------------------------------------------------------------------------ */

enum { K_BITS = 256 };

static u64 cost_model(u64 c, size_t n) {
    u64 windows = (K_BITS + c - 1) / c;
    return windows * ((u64)n + ((u64)1 << c));
}

static u64 best_c(size_t n) {
    u64 best = 4, best_cost = ~(u64)0;
    for (u64 c = 4; c <= 12; ++c) {
        u64 cost = cost_model(c, n);
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

static uint32_t window_digit(const uint8_t* s, size_t bit_offset, u64 c) {
    size_t byte_idx = bit_offset >> 3, bit_in_byte = bit_offset & 7;
    uint32_t word = 0;
    for (int i = 0; i < 4; ++i) {
        size_t bi = byte_idx + (size_t)i;
        if (bi < 32) word |= (uint32_t)s[bi] << (8 * i);
    }
    word >>= bit_in_byte;
    return word & ((1u << c) - 1u);
}

static jac pippenger(const curve* C, const jac* pts, const uint8_t* sc, size_t n) {
    if (n == 0) return jac_zero();
    u64 c = best_c(n);
    size_t M = (size_t)1 << (c - 1);
    size_t chunks = (K_BITS + c - 1) / c;
    jac* buckets = (jac*)malloc(M * sizeof(jac));
    int* carries = (int*)calloc(n, sizeof(int));
    jac* wsum = (jac*)malloc(chunks * sizeof(jac));
    int32_t max_pos = (int32_t)1 << (c - 1);
    for (size_t w = 0; w < chunks; ++w) {
        size_t off = w * c;
        for (size_t k = 0; k < M; ++k) buckets[k] = jac_zero();
        for (size_t i = 0; i < n; ++i) {
            int32_t d = (int32_t)window_digit(sc + 32 * i, off, c) + carries[i];
            carries[i] = 0;
            if (d > max_pos) {
                d -= (int32_t)1 << c;
                carries[i] = 1;
            }
            if (d == 0) continue;
            if (d > 0)
                buckets[d - 1] = jac_add(C, buckets[d - 1], pts[i]);
            else
                buckets[-d - 1] = jac_add(C, buckets[-d - 1], jac_neg(C, pts[i]));
        }
        jac running = jac_zero(), total = jac_zero();
        for (size_t kk = 0; kk < M; ++kk) {
            size_t k = M - 1 - kk;
            running = jac_add(C, running, buckets[k]);
            total = jac_add(C, total, running);
        }
        wsum[w] = total;
    }
    jac result = wsum[chunks - 1];
    for (size_t wi = 1; wi < chunks; ++wi) {
        for (u64 b = 0; b < c; ++b) result = jac_double(C, result);
        result = jac_add(C, result, wsum[chunks - 1 - wi]);
    }
    free(buckets);
    free(carries);
    free(wsum);
    return result;
}

int orc_msm(uint32_t curve_id, const uint8_t* scalars, const uint8_t* points,
            size_t n, uint8_t* result) {
    if (!result) return -1;                          /* GPUKIT_ERR_NULL_ARG */
    if (n > 0 && (!scalars || !points)) return -1;
    const curve* C = curve_by_id(curve_id);
    if (!C) return -3;                               /* GPUKIT_ERR_BACKEND */
    jac* pts = (jac*)malloc((n ? n : 1) * sizeof(jac));
    for (size_t i = 0; i < n; ++i) pts[i] = read_point(C, points + (size_t)C->pt_bytes * i);
    write_point(C, pippenger(C, pts, scalars, n), result);
    free(pts);
    return 0;
}

int orc_msm_naive(uint32_t curve_id, const uint8_t* scalars, const uint8_t* points,
                  size_t n, uint8_t* result) {
    if (!result) return -1;
    if (n > 0 && (!scalars || !points)) return -1;
    const curve* C = curve_by_id(curve_id);
    if (!C) return -3;
    jac acc = jac_zero();
    for (size_t i = 0; i < n; ++i) {
        jac p = read_point(C, points + (size_t)C->pt_bytes * i);
        acc = jac_add(C, acc, jac_mul(C, p, scalars + 32 * i));
    }
    write_point(C, acc, result);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Fr NTT (radix-2 DIT in the order of ntt/cpp/ntt.cpp:128-172).           */
/* ------------------------------------------------------------------------ */

static const field* fr_of(uint32_t curve_id, u64* gen, int* adicity) {
    if (curve_id == ORC_CURVE_BLS12_381) {
        *gen = 7;
        *adicity = 32;
        return &F_BLS_FR;
    }
    if (curve_id == ORC_CURVE_BN254) {
        *gen = 5;
        *adicity = 28;
        return &F_BN_FR;
    }
    return NULL;
}

/* w_n = g^((r-1)/n) in Montgomery form. */
static fe root_mont(const field* F, u64 g, int logn) {
    fe e = F->p;
    e.l[0] -= 1; /* r - 1; r is odd so no borrow */
    for (int s = 0; s < logn; ++s) {
        for (int i = 0; i < F->n; ++i) {
            u64 hi = (i + 1 < F->n) ? e.l[i + 1] : 0;
            e.l[i] = (e.l[i] >> 1) | (hi << 63);
        }
    }
    return f_pow(F, f_from_small(F, g), &e);
}

static int ilog2_exact(size_t n) {
    if (n == 0 || (n & (n - 1))) return -1;
    int l = 0;
    while (((size_t)1 << l) < n) ++l;
    return l;
}

static void bit_reverse(fe* a, size_t n, int logn) {
    for (size_t i = 0; i < n; ++i) {
        size_t j = 0;
        for (int b = 0; b < logn; ++b) j |= ((i >> b) & 1) << (logn - 1 - b);
        if (j > i) {
            fe t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
}

int orc_root_of_unity(uint32_t curve_id, size_t n, uint8_t* out) {
    u64 g;
    int adic;
    const field* F = fr_of(curve_id, &g, &adic);
    int logn = ilog2_exact(n);
    if (!F || logn < 0 || logn > adic) return -2;
    fe w = f_from_mont(F, root_mont(F, g, logn));
    fe_to_le(F, &w, out);
    return 0;
}

int orc_ntt(uint32_t curve_id, uint8_t* data, size_t n, int inverse, int coset) {
    u64 g;
    int adic;
    const field* F = fr_of(curve_id, &g, &adic);
    int logn = ilog2_exact(n);
    if (!F || logn < 0 || logn > adic) return -2;
    fe* a = (fe*)malloc(n * sizeof(fe));
    for (size_t i = 0; i < n; ++i) a[i] = f_to_mont(F, fe_from_le(F, data + 32 * i));
    fe gm = f_from_small(F, g);
    if (coset && !inverse) {
        fe s = f_one(F);
        for (size_t i = 0; i < n; ++i) {
            a[i] = f_mul(F, a[i], s);
            s = f_mul(F, s, gm);
        }
    }
    bit_reverse(a, n, logn);
    for (int s = 1; s <= logn; ++s) {
        size_t m = (size_t)1 << s, half = m >> 1;
        fe wm = root_mont(F, g, s);
        if (inverse) wm = f_inv(F, wm);
        for (size_t k = 0; k < n; k += m) {
            fe w = f_one(F);
            for (size_t j = 0; j < half; ++j) {
                fe u = a[k + j], t = f_mul(F, a[k + j + half], w);
                a[k + j] = f_add(F, u, t);
                a[k + j + half] = f_sub(F, u, t);
                w = f_mul(F, w, wm);
            }
        }
    }
    if (inverse) {
        fe ninv = f_inv(F, f_from_small(F, (u64)n));
        fe gi = f_inv(F, gm), s = ninv;
        for (size_t i = 0; i < n; ++i) {
            a[i] = f_mul(F, a[i], s);
            if (coset) s = f_mul(F, s, gi);
        }
    }
    for (size_t i = 0; i < n; ++i) {
        fe v = f_from_mont(F, a[i]);
        fe_to_le(F, &v, data + 32 * i);
    }
    free(a);
    return 0;
}

int orc_dft(uint32_t curve_id, uint8_t* data, size_t n, int inverse, int coset) {
    u64 g;
    int adic;
    const field* F = fr_of(curve_id, &g, &adic);
    int logn = ilog2_exact(n);
    if (!F || logn < 0 || logn > adic) return -2;
    fe* x = (fe*)malloc(n * sizeof(fe));
    fe* y = (fe*)malloc(n * sizeof(fe));
    for (size_t i = 0; i < n; ++i) x[i] = f_to_mont(F, fe_from_le(F, data + 32 * i));
    fe gm = f_from_small(F, g);
    fe w = root_mont(F, g, logn);
    if (inverse) w = f_inv(F, w);
    if (coset && !inverse) {
        fe s = f_one(F);
        for (size_t i = 0; i < n; ++i) {
            x[i] = f_mul(F, x[i], s);
            s = f_mul(F, s, gm);
        }
    }
    fe wk = f_one(F);
    for (size_t k = 0; k < n; ++k) {
        fe acc, p = f_one(F);
        memset(&acc, 0, sizeof acc);
        for (size_t j = 0; j < n; ++j) {
            acc = f_add(F, acc, f_mul(F, x[j], p));
            p = f_mul(F, p, wk);
        }
        y[k] = acc;
        wk = f_mul(F, wk, w);
    }
    if (inverse) {
        fe ninv = f_inv(F, f_from_small(F, (u64)n));
        fe gi = f_inv(F, gm), s = ninv;
        for (size_t i = 0; i < n; ++i) {
            y[i] = f_mul(F, y[i], s);
            if (coset) s = f_mul(F, s, gi);
        }
    }
    for (size_t i = 0; i < n; ++i) {
        fe v = f_from_mont(F, y[i]);
        fe_to_le(F, &v, data + 32 * i);
    }
    free(x);
    free(y);
    return 0;
}

int orc_fr_powers(uint32_t curve_id, const uint8_t* tau, size_t n, uint8_t* out) {
    u64 g;
    int adic;
    const field* F = fr_of(curve_id, &g, &adic);
    if (!F) return -2;
    fe t = f_to_mont(F, fe_from_le(F, tau)), s = f_one(F);
    for (size_t i = 0; i < n; ++i) {
        fe v = f_from_mont(F, s);
        fe_to_le(F, &v, out + 32 * i);
        s = f_mul(F, s, t);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Compressed BLS12-381 G1 (ZCash/IETF): bit7 compressed, bit6 infinity,    */
/* bit5 set iff y is the lexicographically larger root (y > (p-1)/2).      */
/* Pinned by kzg/test/kzg_test.cpp:38-42 and :64-81.                        */
/* ------------------------------------------------------------------------ */

int orc_g1_compress(const uint8_t* point96, uint8_t* out48) {
    const field* F = &F_BLS_FP;
    int any = 0;
    for (int i = 0; i < 96; ++i) any |= point96[i];
    if (!any) {
        memset(out48, 0, 48);
        out48[0] = 0xC0;
        return 0;
    }
    fe y = fe_from_be(F, point96 + 48);
    fe y2;
    raw_add(F, &y2, &y, &y); /* 2y < 2^384 since y < p < 2^381 */
    memcpy(out48, point96, 48);
    out48[0] |= 0x80;
    if (fe_cmp(F, &y2, &F->p) > 0) out48[0] |= 0x20;
    return 0;
}

int orc_kzg_commit(const uint8_t* evals, size_t n, const uint8_t* srs,
                   uint8_t* commit48) {
    uint8_t* coeffs = (uint8_t*)malloc(32 * (n ? n : 1));
    memcpy(coeffs, evals, 32 * n);
    int rc = orc_ntt(ORC_CURVE_BLS12_381, coeffs, n, 1, 0);
    if (rc) {
        free(coeffs);
        return rc;
    }
    uint8_t pt[96];
    rc = orc_msm(ORC_CURVE_BLS12_381, coeffs, srs, n, pt);
    free(coeffs);
    if (rc) return rc;
    return orc_g1_compress(pt, commit48);
}

/* ---- EIP-2537 G1 MSM (bls/cpp/bls.cpp:194-254, bls/c-abi/c_bls_pairing.cpp:106-110).
 * The reference delegates to blst (absent here); this restates the published
 * EIP-2537 semantics with the definitional checks: each 64-byte coordinate is
 * a big-endian integer below p (so its top 16 bytes are zero), the point is
 * on the curve or is (0,0) = infinity, and the subgroup check is [r]P = O.
 * Infinity entries are dropped, scalars (32 B big-endian) are reduced mod r
 * (exact for points of order r), and the sum comes from orc_msm. */
static int be64_coord_ok(const uint8_t* c) {
    for (int i = 0; i < 16; ++i)
        if (c[i]) return 0;
    fe v = fe_from_be(&F_BLS_FP, c + 16);
    return fe_cmp(&F_BLS_FP, &v, &F_BLS_FP.p) < 0;
}

int orc_bls12_381_g1_msm(uint8_t rx[64], uint8_t ry[64], const uint8_t* xycs, size_t size) {
    if (!rx || !ry || (size && !xycs) || size % 160) return 0;
    const size_t n = size / 160;
    uint8_t* pts = (uint8_t*)malloc(96 * (n ? n : 1));
    uint8_t* scs = (uint8_t*)malloc(32 * (n ? n : 1));
    size_t m = 0;
    uint8_t r_le[32];
    fe_to_le(&F_BLS_FR, &F_BLS_FR.p, r_le);
    for (size_t i = 0; i < n; ++i) {
        const uint8_t* e = xycs + 160 * i;
        if (!be64_coord_ok(e) || !be64_coord_ok(e + 64)) goto invalid;
        uint8_t pt[96];
        memcpy(pt, e + 16, 48);
        memcpy(pt + 48, e + 80, 48);
        if (!orc_g1_on_curve(ORC_CURVE_BLS12_381, pt)) goto invalid;
        int inf = 1;
        for (int k = 0; k < 96; ++k) inf &= pt[k] == 0;
        if (inf) continue;
        uint8_t rp[96];
        orc_g1_mul(ORC_CURVE_BLS12_381, pt, r_le, rp);
        for (int k = 0; k < 96; ++k)
            if (rp[k]) goto invalid;
        /* scalar: big-endian 256-bit -> little-endian, reduced mod r */
        fe s;
        memset(&s, 0, sizeof s);
        for (int k = 0; k < 32; ++k) s.l[k / 8] |= (u64)e[128 + 31 - k] << (8 * (k % 8));
        while (fe_cmp(&F_BLS_FR, &s, &F_BLS_FR.p) >= 0) raw_sub(&F_BLS_FR, &s, &s, &F_BLS_FR.p);
        memcpy(pts + 96 * m, pt, 96);
        fe_to_le(&F_BLS_FR, &s, scs + 32 * m);
        ++m;
    }
    {
        uint8_t out[96];
        memset(out, 0, 96);
        if (m) orc_msm(ORC_CURVE_BLS12_381, scs, pts, m, out);
        memset(rx, 0, 64);
        memset(ry, 0, 64);
        memcpy(rx + 16, out, 48);
        memcpy(ry + 16, out + 48, 48);
    }
    free(pts);
    free(scs);
    return 1;
invalid:
    free(pts);
    free(scs);
    return 0;
}

/* ---- EIP-4844 blob commitment and opening proof (kzg/c-abi/c_kzg_blob.cpp:26-43;
 * the reference calls c-kzg-4844 v2.1.7, absent here).  Restated from the
 * published EIP-4844 definitions by a route independent of the device's:
 * the blob (4096 big-endian elements, element i = p(w^brp(i))) is put in
 * natural order, interpolated to monomial coefficients by the inverse NTT,
 * and committed against a MONOMIAL setup [tau^i]G1 (n x 96 B BE); y = p(z)
 * by Horner; the quotient (p(X) - y)/(X - z) by synthetic division.
 * Returns 0, or -1 if an element or z is not below r. */
#define ORC_BLOB_N 4096

static int blob_to_coeffs(const uint8_t* blob_be, uint8_t* coeffs_le) {
    const field* F = &F_BLS_FR;
    for (uint32_t i = 0; i < ORC_BLOB_N; ++i) {
        fe v = fe_from_be(F, blob_be + 32 * i);
        if (fe_cmp(F, &v, &F->p) >= 0) return -1;
        uint32_t j = 0;
        for (int b = 0; b < 12; ++b) j |= ((i >> b) & 1u) << (11 - b);
        fe_to_le(F, &v, coeffs_le + 32 * j);
    }
    return orc_ntt(ORC_CURVE_BLS12_381, coeffs_le, ORC_BLOB_N, 1, 0) ? -1 : 0;
}

int orc_kzg_blob_commit(const uint8_t* blob_be, const uint8_t* srs, uint8_t commit48[48]) {
    uint8_t* c = (uint8_t*)malloc(32 * ORC_BLOB_N);
    if (blob_to_coeffs(blob_be, c)) {
        free(c);
        return -1;
    }
    uint8_t pt[96];
    orc_msm(ORC_CURVE_BLS12_381, c, srs, ORC_BLOB_N, pt);
    free(c);
    return orc_g1_compress(pt, commit48);
}

int orc_kzg_blob_proof(const uint8_t* blob_be, const uint8_t z_be[32], const uint8_t* srs,
                       uint8_t proof48[48], uint8_t y_be[32]) {
    const field* F = &F_BLS_FR;
    fe z = fe_from_be(F, z_be);
    if (fe_cmp(F, &z, &F->p) >= 0) return -1;
    uint8_t* c = (uint8_t*)malloc(32 * ORC_BLOB_N);
    if (blob_to_coeffs(blob_be, c)) {
        free(c);
        return -1;
    }
    fe zm = f_to_mont(F, z);
    fe* a = (fe*)malloc(ORC_BLOB_N * sizeof(fe));
    for (int k = 0; k < ORC_BLOB_N; ++k) a[k] = f_to_mont(F, fe_from_le(F, c + 32 * k));
    /* synthetic division: q_{k-1} = a_k + z q_k, remainder a_0 + z q_0 = y */
    fe acc = a[ORC_BLOB_N - 1];
    memset(c, 0, 32 * ORC_BLOB_N);
    for (int k = ORC_BLOB_N - 1; k >= 1; --k) {
        fe q = acc; /* q_{k-1} */
        fe qc = f_from_mont(F, q);
        fe_to_le(F, &qc, c + 32 * (k - 1));
        acc = f_add(F, a[k - 1], f_mul(F, zm, q));
    }
    fe y = f_from_mont(F, acc);
    fe_to_be(F, &y, y_be);
    uint8_t pt[96];
    orc_msm(ORC_CURVE_BLS12_381, c, srs, ORC_BLOB_N, pt);
    free(a);
    free(c);
    return orc_g1_compress(pt, proof48);
}

/* ------------------------------------------------------------------------ */
/* Seeded workload inputs, made on the CPU (test and benchmark inputs).      */
/* ------------------------------------------------------------------------ */

/* The xorshift64* streams of the library's kb200_gen_scalars (the generator
 * family of kzg/test/kzg_gpu_determinism_test.cpp:29-36), restated so that
 * the CPU-only legs (the reference arm of the benchmark, the golden-vector
 * script) build the same workload without loading the CUDA library.
 * kind 0: uniform in [0, r) by rejection sampling of 255-bit (BLS12-381) or
 * 254-bit (BN254) draws; kind 1: 25% zero, 25% one, 20% below 2^64, 30%
 * uniform in [0, r). */
typedef struct { u64 x; } xs64;
static u64 xs_next(xs64* g) {
    g->x ^= g->x >> 12;
    g->x ^= g->x << 25;
    g->x ^= g->x >> 27;
    return g->x * 0x2545F4914F6CDD1DULL;
}
static void xs_uniform_fr(xs64* g, const field* R, u64 mask, u64 w[4]) {
    for (;;) {
        for (int i = 0; i < 4; ++i) w[i] = xs_next(g);
        w[3] &= mask;
        fe t;
        memset(&t, 0, sizeof t);
        for (int i = 0; i < 4; ++i) t.l[i] = w[i];
        if (fe_cmp(R, &t, &R->p) < 0) return;
    }
}

int orc_gen_scalars(uint32_t curve_id, uint64_t seed, size_t n, int kind, uint8_t* out) {
    if ((curve_id != ORC_CURVE_BN254 && curve_id != ORC_CURVE_BLS12_381) || (kind != 0 && kind != 1))
        return -1;
    if (!out && n) return -1;
    const field* R = curve_id == ORC_CURVE_BLS12_381 ? &F_BLS_FR : &F_BN_FR;
    const u64 mask = curve_id == ORC_CURVE_BLS12_381 ? 0x7FFFFFFFFFFFFFFFULL : 0x3FFFFFFFFFFFFFFFULL;
    xs64 g = {seed ^ 0x9E3779B97F4A7C15ULL};
    if (g.x == 0) g.x = 0x2545F4914F6CDD1DULL;
    for (size_t i = 0; i < n; ++i) {
        u64 w[4] = {0, 0, 0, 0};
        if (kind == 0) {
            xs_uniform_fr(&g, R, mask, w);
        } else {
            const u64 u = xs_next(&g) % 100;
            if (u < 25) {
            } else if (u < 50) {
                w[0] = 1;
            } else if (u < 70) {
                w[0] = xs_next(&g);
            } else {
                xs_uniform_fr(&g, R, mask, w);
            }
        }
        for (int l = 0; l < 4; ++l)
            for (int b = 0; b < 8; ++b) out[32 * i + 8 * l + b] = (uint8_t)(w[l] >> (8 * b));
    }
    return 0;
}

/* Fixed-base k_i * G for many scalars: 8-bit windows over a table of
 * d * 2^(8w) * G (d < 256, w < 32, affine Montgomery), one mixed Jacobian
 * addition per non-zero byte, then one batched affine normalisation
 * (Montgomery's trick) per block of outputs.  The result is the unique
 * affine point k_i * G, so it equals every other correct route (the
 * double-and-add of orc_g1_mul_gen, the reference ladder, the device
 * fixed-base kernel) byte for byte. */
#include <pthread.h>

typedef struct { fe x, y; } aff;

/* madd-2007-bl (Z2 = 1); equal or opposite operands fall back to the
 * complete formulas above. */
static jac jac_add_affine(const curve* C, jac a, const aff* q) {
    const field* F = C->F;
    if (a.inf) {
        jac r = {q->x, q->y, f_one(F), 0};
        return r;
    }
    fe Z1Z1 = f_sqr(F, a.Z);
    fe U2 = f_mul(F, q->x, Z1Z1);
    fe S2 = f_mul(F, f_mul(F, q->y, a.Z), Z1Z1);
    fe H = f_sub(F, U2, a.X);
    if (fe_is_zero(F, &H)) {
        jac b = {q->x, q->y, f_one(F), 0};
        return jac_add(C, a, b);
    }
    fe HH = f_sqr(F, H);
    fe I = f_add(F, HH, HH);
    I = f_add(F, I, I);
    fe J = f_mul(F, H, I);
    fe rr = f_sub(F, S2, a.Y);
    rr = f_add(F, rr, rr);
    fe V = f_mul(F, a.X, I);
    fe X3 = f_sub(F, f_sub(F, f_sqr(F, rr), J), f_add(F, V, V));
    fe Y1J = f_mul(F, a.Y, J);
    fe Y3 = f_sub(F, f_mul(F, rr, f_sub(F, V, X3)), f_add(F, Y1J, Y1J));
    fe Z3 = f_sub(F, f_sub(F, f_sqr(F, f_add(F, a.Z, H)), Z1Z1), HH);
    jac out = {X3, Y3, Z3, 0};
    return out;
}

static aff* g_fb_table[3];  /* by curve id; 32 x 256 entries (entry 0 unused) */
static pthread_mutex_t g_fb_mu = PTHREAD_MUTEX_INITIALIZER;

static void to_affine_batch(const curve* C, jac* P, size_t m, aff* out, int* inf, fe* scratch) {
    const field* F = C->F;
    fe acc = f_one(F);
    for (size_t i = 0; i < m; ++i) {
        inf[i] = P[i].inf || fe_is_zero(F, &P[i].Z);
        scratch[i] = acc;
        if (!inf[i]) acc = f_mul(F, acc, P[i].Z);
    }
    fe inv = f_inv(F, acc);
    for (size_t i = m; i-- > 0;) {
        if (inf[i]) continue;
        fe zi = f_mul(F, inv, scratch[i]);
        inv = f_mul(F, inv, P[i].Z);
        fe zi2 = f_sqr(F, zi);
        out[i].x = f_mul(F, P[i].X, zi2);
        out[i].y = f_mul(F, P[i].Y, f_mul(F, zi2, zi));
    }
}

static const aff* fixed_base_table(const curve* C, uint32_t curve_id) {
    pthread_mutex_lock(&g_fb_mu);
    if (!g_fb_table[curve_id]) {
        const size_t m = 32 * 256;
        jac* P = (jac*)calloc(m, sizeof(jac));
        aff* T = (aff*)calloc(m, sizeof(aff));
        int* inf = (int*)calloc(m, sizeof(int));
        fe* scr = (fe*)calloc(m, sizeof(fe));
        jac base = generator(C);
        for (int w = 0; w < 32; ++w) {
            P[w * 256] = jac_zero();
            for (int d = 1; d < 256; ++d) P[w * 256 + d] = jac_add(C, P[w * 256 + d - 1], base);
            for (int k = 0; k < 8; ++k) base = jac_double(C, base);
        }
        to_affine_batch(C, P, m, T, inf, scr);
        free(P);
        free(inf);
        free(scr);
        g_fb_table[curve_id] = T;
    }
    pthread_mutex_unlock(&g_fb_mu);
    return g_fb_table[curve_id];
}

typedef struct {
    const curve* C;
    const aff* T;
    const uint8_t* k;
    uint8_t* out;
    size_t lo, hi;
} fb_job;

static void* fb_worker(void* arg) {
    fb_job* j = (fb_job*)arg;
    const curve* C = j->C;
    const field* F = C->F;
    enum { BLK = 2048 };
    jac* P = (jac*)malloc(BLK * sizeof(jac));
    aff* A = (aff*)malloc(BLK * sizeof(aff));
    int* inf = (int*)malloc(BLK * sizeof(int));
    fe* scr = (fe*)malloc(BLK * sizeof(fe));
    for (size_t b = j->lo; b < j->hi; b += BLK) {
        const size_t m = (j->hi - b) < BLK ? (j->hi - b) : BLK;
        for (size_t i = 0; i < m; ++i) {
            const uint8_t* k = j->k + 32 * (b + i);
            jac acc = jac_zero();
            for (int w = 0; w < 32; ++w)
                if (k[w]) acc = jac_add_affine(C, acc, &j->T[w * 256 + k[w]]);
            P[i] = acc;
        }
        to_affine_batch(C, P, m, A, inf, scr);
        for (size_t i = 0; i < m; ++i) {
            uint8_t* o = j->out + (size_t)C->pt_bytes * (b + i);
            if (inf[i]) {
                memset(o, 0, (size_t)C->pt_bytes);
                continue;
            }
            fe x = f_from_mont(F, A[i].x), y = f_from_mont(F, A[i].y);
            fe_to_be(F, &x, o);
            fe_to_be(F, &y, o + F->bytes);
        }
    }
    free(P);
    free(A);
    free(inf);
    free(scr);
    return NULL;
}

int orc_g1_fixed_base_batch(uint32_t curve_id, const uint8_t* scalars_le, size_t n,
                            uint8_t* out, int threads) {
    const curve* C = curve_by_id(curve_id);
    if (!C || ((!scalars_le || !out) && n)) return -1;
    if (n == 0) return 0;
    const aff* T = fixed_base_table(C, curve_id);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if ((size_t)threads > n) threads = (int)n;
    pthread_t th[256];
    fb_job jobs[256];
    for (int t = 0; t < threads; ++t) {
        jobs[t].C = C;
        jobs[t].T = T;
        jobs[t].k = scalars_le;
        jobs[t].out = out;
        jobs[t].lo = n * (size_t)t / (size_t)threads;
        jobs[t].hi = n * (size_t)(t + 1) / (size_t)threads;
        if (pthread_create(&th[t], NULL, fb_worker, &jobs[t]) != 0) {
            fb_worker(&jobs[t]);
            th[t] = 0;
        }
    }
    for (int t = 0; t < threads; ++t)
        if (th[t]) pthread_join(th[t], NULL);
    return 0;
}
