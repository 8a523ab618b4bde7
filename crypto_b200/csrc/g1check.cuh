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

// Jacobian coordinates (x, y) = (X / Z^2, Y / Z^3) on y^2 = x^3 + 4; Z = 0 is
// infinity.  The membership test below runs two 64-bit double-and-add chains
// per point, so it uses the a = 0 doubling of 7 products (against 9 for an
// XYZZ doubling).
struct G1Jac {
    Fe<FpBLS> X, Y, Z;
};

__device__ __forceinline__ void g1j_set_inf(G1Jac& p) {
    fe_one(p.X);
    fe_one(p.Y);
    fe_zero(p.Z);
}

// dbl-2009-l (a = 0): A = X^2, B = Y^2, C = B^2, D = 2((X + B)^2 - A - C),
// E = 3A, X3 = E^2 - 2D, Y3 = E(D - X3) - 8C, Z3 = 2YZ.  Infinity stays
// infinity (Z3 = 0).
__device__ __forceinline__ void g1j_dbl(G1Jac& p) {
    using F = FpBLS;
    Fe<F> A, B, C, D, E, t;
    fe_sqr(A, p.X);
    fe_sqr(B, p.Y);
    fe_sqr(C, B);
    fe_add(t, p.X, B);
    fe_sqr(D, t);
    fe_sub(D, D, A);
    fe_sub(D, D, C);
    fe_dbl(D, D);
    fe_dbl(E, A);
    fe_add(E, E, A);
    fe_mul(p.Z, p.Y, p.Z);
    fe_dbl(p.Z, p.Z);
    fe_sqr(t, E);
    fe_sub(t, t, D);
    fe_sub(p.X, t, D);
    fe_sub(t, D, p.X);
    fe_mul(t, E, t);
    fe_dbl(C, C);
    fe_dbl(C, C);
    fe_dbl(C, C);
    fe_sub(p.Y, t, C);
}

// The same doubling with its independent products issued in inlined pairs
// (A and B, C and the square of X + B, YZ and E^2), so each pair's
// instruction streams interleave; the membership test inlines it once.
// EIP-2537 MSM at 2^16: 7.65 -> 7.17 ms.
__device__ __forceinline__ void g1j_dbl_ilp(G1Jac& p) {
    using F = FpBLS;
    Fe<F> A, B, C, D, E, t, zn;
    fe_mul_inl(A, p.X, p.X);
    fe_mul_inl(B, p.Y, p.Y);
    fe_add(t, p.X, B);
    fe_mul_inl(C, B, B);
    fe_mul_inl(D, t, t);
    fe_sub(D, D, A);
    fe_sub(D, D, C);
    fe_dbl(D, D);
    fe_dbl(E, A);
    fe_add(E, E, A);
    fe_mul_inl(zn, p.Y, p.Z);
    fe_mul_inl(t, E, E);
    fe_dbl(p.Z, zn);
    fe_sub(t, t, D);
    fe_sub(p.X, t, D);
    fe_sub(t, D, p.X);
    fe_mul(t, E, t);
    fe_dbl(C, C);
    fe_dbl(C, C);
    fe_dbl(C, C);
    fe_sub(p.Y, t, C);
}

// madd-2007-bl: p += a for a finite affine point a (11 products).
__device__ __forceinline__ void g1j_madd(G1Jac& p, const Affine<FpBLS>& a) {
    using F = FpBLS;
    if (fe_is_zero(p.Z)) {
        p.X = a.x;
        p.Y = a.y;
        fe_one(p.Z);
        return;
    }
    Fe<F> Z1Z1, H, r, HH, I, J, V, t;
    fe_sqr(Z1Z1, p.Z);
    fe_mul(H, a.x, Z1Z1);
    fe_sub(H, H, p.X);          // H = x2 Z1^2 - X1
    fe_mul(t, p.Z, Z1Z1);
    fe_mul(t, a.y, t);
    fe_sub(r, t, p.Y);
    fe_dbl(r, r);               // r = 2 (y2 Z1^3 - Y1)
    if (fe_is_zero(H)) {
        if (fe_is_zero(r))
            g1j_dbl(p);
        else
            g1j_set_inf(p);
        return;
    }
    fe_sqr(HH, H);
    fe_dbl(I, HH);
    fe_dbl(I, I);               // I = 4 HH
    fe_mul(J, H, I);
    fe_mul(V, p.X, I);
    fe_add(t, p.Z, H);
    fe_sqr(t, t);
    fe_sub(t, t, Z1Z1);
    fe_sub(p.Z, t, HH);         // Z3 = (Z1 + H)^2 - Z1Z1 - HH
    fe_sqr(t, r);
    fe_sub(t, t, J);
    fe_sub(t, t, V);
    fe_sub(t, t, V);            // X3 = r^2 - J - 2V
    fe_sub(V, V, t);
    fe_mul(V, r, V);
    fe_mul(J, p.Y, J);
    fe_dbl(J, J);
    fe_sub(p.Y, V, J);          // Y3 = r (V - X3) - 2 Y1 J
    p.X = t;
}

// add-2007-bl: p += q for a finite Jacobian q with qzz = Zq^2 and
// qzzz = Zq^3 precomputed (14 products).
__device__ __forceinline__ void g1j_add_cached(G1Jac& p, const G1Jac& q, const Fe<FpBLS>& qzz,
                                               const Fe<FpBLS>& qzzz) {
    using F = FpBLS;
    if (fe_is_zero(p.Z)) {
        p = q;
        return;
    }
    Fe<F> Z1Z1, U1, S1, H, r, I, J, V, t;
    fe_sqr(Z1Z1, p.Z);
    fe_mul(U1, p.X, qzz);
    fe_mul(H, q.X, Z1Z1);
    fe_sub(H, H, U1);           // H = U2 - U1
    fe_mul(S1, p.Y, qzzz);
    fe_mul(t, p.Z, Z1Z1);
    fe_mul(t, q.Y, t);
    fe_sub(r, t, S1);
    fe_dbl(r, r);               // r = 2 (S2 - S1)
    if (fe_is_zero(H)) {
        if (fe_is_zero(r))
            g1j_dbl(p);
        else
            g1j_set_inf(p);
        return;
    }
    fe_dbl(I, H);
    fe_sqr(I, I);               // I = (2H)^2
    fe_mul(J, H, I);
    fe_mul(V, U1, I);
    fe_add(t, p.Z, q.Z);
    fe_sqr(t, t);
    fe_sub(t, t, Z1Z1);
    fe_sub(t, t, qzz);
    fe_mul(p.Z, t, H);          // Z3 = ((Z1 + Z2)^2 - Z1Z1 - Z2Z2) H
    fe_sqr(t, r);
    fe_sub(t, t, J);
    fe_sub(t, t, V);
    fe_sub(t, t, V);            // X3 = r^2 - J - 2V
    fe_sub(V, V, t);
    fe_mul(V, r, V);
    fe_mul(J, S1, J);
    fe_dbl(J, J);
    fe_sub(p.Y, V, J);          // Y3 = r (V - X3) - 2 S1 J
    p.X = t;
}

// A finite affine point on the curve (Montgomery form) is in G1 iff
// sigma(P) = -[u^2]P (M. Scott, "A note on group membership tests for G1,
// G2 and GT on BLS pairing-friendly curves", 2021): two [|u|] chains
// (double-and-add from the top bit; bit 63 of |u| is set), the first with
// affine additions of P, the second with additions of the first's result,
// run as one loop so the doubling's body appears once.
static __device__ __noinline__ bool g1_in_subgroup(const Affine<FpBLS>& a) {
    using F = FpBLS;
    G1Jac q1, q2;
    q2.X = a.x;
    q2.Y = a.y;
    fe_one(q2.Z);
    Fe<F> qzz, qzzz;
    for (int it = 0; it < 126; ++it) {
        if (it == 63) {
            if (fe_is_zero(q2.Z)) return false;  // [|u|]P = O: P is torsion outside G1
            q1 = q2;
            fe_sqr(qzz, q1.Z);
            fe_mul(qzzz, qzz, q1.Z);
        }
        const int b = 62 - (it < 63 ? it : it - 63);
        g1j_dbl_ilp(q2);
        if ((BLS_U_ABS >> b) & 1ull) {
            if (it < 63)
                g1j_madd(q2, a);
            else
                g1j_add_cached(q2, q1, qzz, qzzz);
        }
    }
    if (fe_is_zero(q2.Z)) return false;
    Fe<F> beta, t, zz;
    fe_sqr(zz, q2.Z);
    fe_load(beta, kG1Beta);
    fe_to_mont(beta, beta);
    fe_mul(t, beta, a.x);
    fe_mul(t, t, zz);
    if (!fe_eq(t, q2.X)) return false;  // beta x == X / Z^2
    fe_mul(zz, zz, q2.Z);
    fe_neg(t, a.y);
    fe_mul(t, t, zz);
    return fe_eq(t, q2.Y);              // -y == Y / Z^3
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
