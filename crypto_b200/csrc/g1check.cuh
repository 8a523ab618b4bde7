// Validity checks for BLS12-381 G1 input points, shared by the EIP-2537 MSM
// input path and the blob-setup loader: canonical range, curve equation and
// G1 membership.
#pragma once
#include "curve.cuh"

namespace kb200 {

// |u| for the BLS12-381 parameter u = -0xd201000000010000.
constexpr uint64_t BLS_U_ABS = 0xd201000000010000ull;

// beta: the primitive cube root of unity of Fp for which
// sigma(x, y) = (beta x, y) acts on G1 as multiplication by -u^2
// (canonical, little-endian 32-bit words).
static __constant__ uint32_t kG1Beta[12] = {0xfffefffe, 0x2e01ffff, 0x620a0002, 0xde17d813,
                                     0xe6f89688, 0xddb3a93b, 0x6a0f77ea, 0xba69c607,
                                     0xdf76ce51, 0x5f19672f, 0x00000000, 0x00000000};

template <class Fx>
__device__ __forceinline__ bool below_modulus(const Fe<Fx>& a) {
    for (int i = Fx::N - 1; i >= 0; --i) {
        if (a.v[i] != Fx::P(i)) return a.v[i] < Fx::P(i);
    }
    return false;
}

// [|u|] base, double-and-add from the top bit (bit 63 is set).
__device__ __forceinline__ void g1_mul_abs_u(Xyzz<FpBLS>& acc, const Xyzz<FpBLS>& base) {
    acc = base;
    for (int b = 62; b >= 0; --b) {
        xyzz_dbl(acc, acc);
        if ((BLS_U_ABS >> b) & 1ull) xyzz_add(acc, base);
    }
}

// A finite affine point on the curve (Montgomery form) is in G1 iff
// sigma(P) = -[u^2]P (M. Scott, "A note on group membership tests for G1,
// G2 and GT on BLS pairing-friendly curves", 2021).
static __device__ __noinline__ bool g1_in_subgroup(const Affine<FpBLS>& a) {
    using F = FpBLS;
    Xyzz<F> p, q1, q2;
    xyzz_from_affine(p, a);
    g1_mul_abs_u(q1, p);
    g1_mul_abs_u(q2, q1);  // [u^2] P
    if (xyzz_is_inf(q2)) return false;
    Fe<F> beta, t;
    fe_load(beta, kG1Beta);
    fe_to_mont(beta, beta);
    fe_mul(t, beta, a.x);
    fe_mul(t, t, q2.ZZ);
    if (!fe_eq(t, q2.X)) return false;  // beta x == X / ZZ
    fe_neg(t, a.y);
    fe_mul(t, t, q2.ZZZ);
    return fe_eq(t, q2.Y);              // -y == Y / ZZZ
}

// y^2 == x^3 + 4 (Montgomery form).
__device__ __forceinline__ bool g1_on_curve(const Affine<FpBLS>& a) {
    using F = FpBLS;
    Fe<F> l, r, b;
    fe_sqr(l, a.y);
    fe_sqr(r, a.x);
    fe_mul(r, r, a.x);
    fe_one(b);
    fe_add(b, b, b);
    fe_add(b, b, b);  // 4
    fe_add(r, r, b);
    return fe_eq(l, r);
}

}  // namespace kb200
