// G1 group arithmetic on device for the two a = 0 short-Weierstrass curves:
//   BLS12-381 G1 : y^2 = x^3 + 4 over FpBLS   (bls/cpp/bls12_381_g1.hpp)
//   BN254 G1     : y^2 = x^3 + 3 over FpBN    (bn254/cpp/bn254_g1.hpp)
//
// Coordinates: accumulators are extended Jacobian "XYZZ" points
// (x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2, infinity <=> ZZ = 0), using the
// published Explicit-Formulas-Database formulas madd-2008-s, add-2008-s,
// dbl-2008-s-1 and mdbl-2008-s-1 for a = 0.  Inputs are affine points in
// Montgomery form.  Exceptional cases (P = Q, P = -Q, infinity operands) are
// handled explicitly, so every result is the exact group element; the final
// affine encoding is therefore identical to the reference's Jacobian path.
#pragma once
#include "field.cuh"

namespace kb200 {

// Resident 128-thread blocks per SM requested for the bucket-accumulation
// kernel (sets its register budget: 5 -> 96 registers, 6 -> 80).
#ifndef KB_ACC_MIN_BLOCKS_BLS
#define KB_ACC_MIN_BLOCKS_BLS 5
#endif
#ifndef KB_ACC_MIN_BLOCKS_BN
#define KB_ACC_MIN_BLOCKS_BN 6
#endif

struct G1BLS {
    using F = FpBLS;
    static constexpr uint32_t B = 4;
    static constexpr int WIRE = 96;  // x || y, 48-byte big-endian each
    static constexpr int CURVE_ID = 2;
    static constexpr int ACC_MIN_BLOCKS = KB_ACC_MIN_BLOCKS_BLS;
};
// GLV endomorphism of BLS12-381 G1: phi(x, y) = (beta2 x, y) = [lambda](x, y)
// for lambda = u^2 - 1, with beta2 = 0x1a0111ea397fe699ec024086...0000aaac
// (a cube root of unity mod p), here in Montgomery form (beta2 * 2^384 mod p).
static __constant__ uint32_t kGlvBeta2Mont[12] = {0x8671f071, 0xcd03c9e4, 0x1fcda5d2, 0x5dab2246,
                                                  0xd3851b95, 0x587042af, 0x01bacb9e, 0x8eb60ebe,
                                                  0x83d050d2, 0x03f97d6e, 0x54638741, 0x18f02065};

// GLV endomorphism of BN254 G1: phi(x, y) = (beta x, y) = [lambda](x, y)
// with lambda = 0xb3c4d79d41a917585bfc41088d8daaa78b17ea66b99c90dd (a cube
// root of unity mod r) and beta = 0x59e26bcea0d48bacd4f263f1acdb5c4f5763473177fffffe
// (a cube root of unity mod p; the pair is matched on the generator), here
// in Montgomery form (beta * 2^256 mod p).  Every BN254 point has order r
// (cofactor 1), so the identity holds for every input point.
static __constant__ uint32_t kBnGlvBetaMont[8] = {0xd782e155, 0x71930c11, 0xffbe3323, 0xa6bb947c,
                                                  0xd4741444, 0xaa303344, 0x26594943, 0x2c3b3f0d};

struct G1BN {
    using F = FpBN;
    static constexpr uint32_t B = 3;
    static constexpr int WIRE = 64;  // x || y, 32-byte big-endian each
    static constexpr int CURVE_ID = 1;
    static constexpr int ACC_MIN_BLOCKS = KB_ACC_MIN_BLOCKS_BN;
};

template <class F>
struct Affine {
    Fe<F> x, y;
};
template <class F>
struct Xyzz {
    Fe<F> X, Y, ZZ, ZZZ;
};

// Internal affine table entries are 2N words (x then y, Montgomery form).
// The top bit of x's most significant word flags the point at infinity; it
// is free because every modulus here is below 2^(32N - 1).
constexpr uint32_t INF_FLAG = 0x80000000u;

template <class F>
KB_DEV bool aff_is_inf_words(const uint32_t* w) {
    return (w[F::N - 1] & INF_FLAG) != 0;
}

template <class F>
KB_DEV void xyzz_set_inf(Xyzz<F>& p) {
    fe_zero(p.X);
    fe_zero(p.Y);
    fe_zero(p.ZZ);
    fe_zero(p.ZZZ);
}
template <class F>
KB_DEV bool xyzz_is_inf(const Xyzz<F>& p) {
    return fe_is_zero(p.ZZ);
}
template <class F>
KB_DEV void xyzz_from_affine(Xyzz<F>& p, const Affine<F>& a) {
    p.X = a.x;
    p.Y = a.y;
    fe_one(p.ZZ);
    fe_one(p.ZZZ);
}

// dbl-2008-s-1 with a = 0.
template <class F>
KB_DEV void xyzz_dbl(Xyzz<F>& r, const Xyzz<F>& p) {
    Fe<F> U, V, W, S, M, t;
    fe_dbl(U, p.Y);
    fe_sqr(V, U);
    fe_mul(W, U, V);
    fe_mul(S, p.X, V);
    fe_sqr(t, p.X);
    fe_dbl(M, t);
    fe_add(M, M, t);
    Fe<F> X3, Y3;
    fe_sqr(X3, M);
    fe_sub(X3, X3, S);
    fe_sub(X3, X3, S);
    fe_sub(t, S, X3);
    fe_mul(Y3, M, t);
    fe_mul(t, W, p.Y);
    fe_sub(Y3, Y3, t);
    fe_mul(r.ZZ, V, p.ZZ);
    fe_mul(r.ZZZ, W, p.ZZZ);
    r.X = X3;
    r.Y = Y3;
}

// dbl-2008-s-1 with the products inlined: for long serial doubling chains
// (window combine), where one inlined copy in a loop beats a call per product.
template <class F>
KB_DEV void xyzz_dbl_inl(Xyzz<F>& p) {
    Fe<F> U, V, W, S, M, t;
    fe_dbl(U, p.Y);
    fe_sqr_inl(V, U);
    fe_mul_inl(W, U, V);
    fe_mul_inl(S, p.X, V);
    fe_sqr_inl(t, p.X);
    fe_dbl(M, t);
    fe_add(M, M, t);
    fe_mul_inl(p.ZZ, V, p.ZZ);
    fe_mul_inl(p.ZZZ, W, p.ZZZ);
    fe_mul_inl(W, W, p.Y);
    fe_sqr_inl(p.X, M);
    fe_sub(p.X, p.X, S);
    fe_sub(p.X, p.X, S);
    fe_sub(t, S, p.X);
    fe_mul_inl(p.Y, M, t);
    fe_sub(p.Y, p.Y, W);
}

// Lane k's copy of a field element, for every lane of the warp.
template <class F>
KB_DEV void fe_bcast(Fe<F>& r, const Fe<F>& a, int k) {
#pragma unroll
    for (int i = 0; i < F::N; ++i) r.v[i] = __shfl_sync(0xffffffffu, a.v[i], k);
}

// dbl-2008-s-1 with the products spread over the lanes of a full warp: every
// lane holds the same point; each of the three stages runs its independent
// products on lanes 0..3 at once and broadcasts them, so a doubling costs
// three product latencies on the critical path instead of nine.  For long
// serial doubling chains (window weighting).  All 32 lanes must call it.
template <class F>
KB_DEV void xyzz_dbl_warp(Xyzz<F>& p) {
    const int lane = threadIdx.x & 31;
    Fe<F> U, a, b, r;
    fe_dbl(U, p.Y);
    // stage 1: V = U^2 (lane 0), t = X^2 (lane 1)
    a = lane == 1 ? p.X : U;
    fe_mul_inl(r, a, a);
    Fe<F> V, t, M;
    fe_bcast(V, r, 0);
    fe_bcast(t, r, 1);
    fe_dbl(M, t);
    fe_add(M, M, t);
    // stage 2: W = U V (0), S = X V (1), ZZ3 = V ZZ (2), M^2 (3)
    a = lane == 1 ? p.X : (lane == 2 ? p.ZZ : (lane == 3 ? M : U));
    b = lane == 3 ? M : V;
    fe_mul_inl(r, a, b);
    Fe<F> W, S, M2;
    fe_bcast(W, r, 0);
    fe_bcast(S, r, 1);
    fe_bcast(p.ZZ, r, 2);
    fe_bcast(M2, r, 3);
    fe_sub(p.X, M2, S);
    fe_sub(p.X, p.X, S);  // X3 = M^2 - 2S
    fe_sub(S, S, p.X);
    // stage 3: M (S - X3) (0), W Y (1), W ZZZ (2)
    a = lane == 0 ? M : W;
    b = lane == 0 ? S : (lane == 1 ? p.Y : p.ZZZ);
    fe_mul_inl(r, a, b);
    Fe<F> Ya, WY;
    fe_bcast(Ya, r, 0);
    fe_bcast(WY, r, 1);
    fe_bcast(p.ZZZ, r, 2);
    fe_sub(p.Y, Ya, WY);  // Y3 = M(S - X3) - W Y
}

// dbl-2008-s-1 on a point held in shared memory (X, Y, ZZ, ZZZ as 4N
// consecutive words), the products spread over lanes 0..3 of the warp like
// xyzz_dbl_warp, with every operand and result passing through shared memory
// (tmp: 7N words of scratch) so that no lane holds the point in registers:
// for kernels whose register budget is tight.  All 32 lanes must call it.
template <class F>
KB_DEV void xyzz_dbl_warp_sm(uint32_t* p, uint32_t* tmp) {
    constexpr int N = F::N;
    const int lane = threadIdx.x & 31;
    uint32_t* pX = p;
    uint32_t* pY = p + N;
    uint32_t* pZZ = p + 2 * N;
    uint32_t* pZZZ = p + 3 * N;
    uint32_t* tU = tmp;
    uint32_t* tV = tmp + N;
    uint32_t* tM = tmp + 2 * N;
    uint32_t* tW = tmp + 3 * N;
    uint32_t* tS = tmp + 4 * N;
    uint32_t* tM2 = tmp + 5 * N;
    uint32_t* tWY = tmp + 6 * N;
    Fe<F> a, b, r;
    // stage 1: V = U^2 with U = 2Y (lane 0), X^2 -> M = 3 X^2 (lane 1)
    fe_load(a, lane == 1 ? pX : pY);
    fe_dbl(b, a);
#pragma unroll
    for (int i = 0; i < N; ++i) a.v[i] = lane == 1 ? a.v[i] : b.v[i];
    fe_mul_inl(r, a, a);
    if (lane == 0) {
        fe_store(tU, a);
        fe_store(tV, r);
    } else if (lane == 1) {
        fe_dbl(b, r);
        fe_add(b, b, r);
        fe_store(tM, b);
    }
    __syncwarp();
    // stage 2: W = U V (0), S = X V (1), ZZ3 = V ZZ (2), M^2 (3)
    fe_load(a, lane == 1 ? pX : (lane == 2 ? pZZ : (lane == 3 ? tM : tU)));
    fe_load(b, lane == 3 ? tM : tV);
    fe_mul_inl(r, a, b);
    if (lane < 4) fe_store(lane == 1 ? tS : (lane == 2 ? pZZ : (lane == 3 ? tM2 : tW)), r);
    __syncwarp();
    // stage 3: M (S - X3) (0), W Y (1), W ZZZ (2), with X3 = M^2 - 2S
    Fe<F> X3, Sd;
    fe_load(a, tM2);
    fe_load(Sd, tS);
    fe_sub(X3, a, Sd);
    fe_sub(X3, X3, Sd);
    fe_sub(Sd, Sd, X3);
    if (lane == 0) fe_store(pX, X3);  // nothing reads X in this stage
    fe_load(a, lane == 0 ? tM : tW);
    fe_load(b, lane == 2 ? pZZZ : pY);  // only lane 2 reads what it rewrites
#pragma unroll
    for (int i = 0; i < N; ++i) b.v[i] = lane == 0 ? Sd.v[i] : b.v[i];
    fe_mul_inl(r, a, b);
    if (lane == 1) fe_store(tWY, r);
    if (lane == 2) fe_store(pZZZ, r);
    __syncwarp();
    // Y3 = M (S - X3) - W Y
    if (lane == 0) {
        fe_load(a, tWY);
        fe_sub(r, r, a);
        fe_store(pY, r);
    }
    __syncwarp();
}

// k >= 0 doublings of a point in shared memory (4N words: X, Y, ZZ, ZZZ)
// with the coordinates dbl-2008-s-1 gives, two product levels per doubling
// instead of three: the chain carries X^2, 3X^3 and 2Y^2 beside the point.
// With t = 3X^3 - 2Y^2 and u = 3t - 2Y^2 (= 9X^3 - 8Y^2), the Jacobian
// doubling for a = 0 (X' = 9X^4 - 8XY^2, Y' = 36X^3Y^2 - 27X^6 - 8Y^4,
// Z' = 2YZ, with ZZ = Z^2 and ZZZ = Z^3) reads
//   X' = X u,  Y' = 2 (2Y^2 t) - 3X^3 u,  ZZ' = 2 (ZZ 2Y^2),  ZZZ' = 4 ((Y 2Y^2) ZZZ),
//   X'^2 = X^2 u^2,  3X'^3 = (3X^3 u) u^2,  2Y'^2 = (2Y') Y',
// level 1 on lanes 0..5 (X u, u^2, 3X^3 u, 2Y^2 t, Y 2Y^2, ZZ 2Y^2), level 2
// on lanes 0..3.  tmp: 8N words of shared scratch.  All 32 lanes call it.
template <class F>
KB_DEV void xyzz_dbl_chain_warp_sm(uint32_t* p, uint32_t k, uint32_t* tmp) {
    constexpr int N = F::N;
    const int lane = threadIdx.x & 31;
    if (k == 0) return;
    uint32_t* pX = p;
    uint32_t* pY = p + N;
    uint32_t* pZZ = p + 2 * N;
    uint32_t* pZZZ = p + 3 * N;
    uint32_t* tX2 = tmp;          // X^2
    uint32_t* tX3 = tmp + N;      // 3 X^3
    uint32_t* tY2 = tmp + 2 * N;  // 2 Y^2
    uint32_t* tXn = tmp + 3 * N;  // X u = X'
    uint32_t* tU2 = tmp + 4 * N;  // u^2
    uint32_t* tVU = tmp + 5 * N;  // 3 X^3 u
    uint32_t* tT = tmp + 6 * N;   // 2 Y^2 t
    uint32_t* tY3 = tmp + 7 * N;  // Y 2Y^2
    Fe<F> a, b, r, c;
    // set-up: X^2 (lane 0), Y^2 (lane 1); then X X^2 (lane 0)
    fe_load(a, lane == 1 ? pY : pX);
    fe_mul_inl(r, a, a);
    if (lane == 0) fe_store(tX2, r);
    if (lane == 1) {
        fe_dbl(r, r);
        fe_store(tY2, r);
    }
    __syncwarp();
    fe_load(a, pX);
    fe_load(b, tX2);
    fe_mul_inl(r, a, b);
    if (lane == 0) {
        fe_dbl(c, r);
        fe_add(r, c, r);
        fe_store(tX3, r);
    }
    __syncwarp();
    for (uint32_t it = 0; it < k; ++it) {
        Fe<F> t, u, y2;
        fe_load(c, tX3);
        fe_load(y2, tY2);
        fe_sub(t, c, y2);
        fe_dbl(u, t);
        fe_add(u, u, t);
        fe_sub(u, u, y2);
        // level 1 (lanes that compute nothing read tX3, which no lane writes here)
        fe_load(a, lane == 0 ? pX
                             : (lane == 3 ? tY2 : (lane == 4 ? pY : (lane == 5 ? pZZ : tX3))));
#pragma unroll
        for (int i = 0; i < N; ++i) {
            a.v[i] = lane == 1 ? u.v[i] : a.v[i];
            b.v[i] = lane <= 2 ? u.v[i] : (lane == 3 ? t.v[i] : y2.v[i]);
        }
        fe_mul_inl(r, a, b);
        if (lane == 0) fe_store(tXn, r);
        if (lane == 1) fe_store(tU2, r);
        if (lane == 2) fe_store(tVU, r);
        if (lane == 3) fe_store(tT, r);
        if (lane == 4) fe_store(tY3, r);
        if (lane == 5) {
            fe_dbl(r, r);
            fe_store(pZZ, r);  // ZZ' = 2 (ZZ 2Y^2); only lane 5 reads ZZ
        }
        __syncwarp();
        // Y' = 2 (2Y^2 t) - 3X^3 u and 2Y'
        Fe<F> yn, yd;
        fe_load(a, tT);
        fe_load(b, tVU);
        fe_dbl(yn, a);
        fe_sub(yn, yn, b);
        fe_dbl(yd, yn);
        // level 2
        fe_load(a, lane == 0 ? tX2 : (lane == 3 ? tY3 : tVU));
        fe_load(b, lane == 3 ? pZZZ : tU2);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            a.v[i] = lane == 2 ? yd.v[i] : a.v[i];
            b.v[i] = lane == 2 ? yn.v[i] : b.v[i];
        }
        fe_mul_inl(r, a, b);
        if (lane == 0) fe_store(tX2, r);
        if (lane == 1) fe_store(tX3, r);
        if (lane == 2) fe_store(tY2, r);
        if (lane == 3) {
            fe_dbl(r, r);
            fe_dbl(r, r);
            fe_store(pZZZ, r);
        }
        if (lane == 4) {
            fe_load(c, tXn);
            fe_store(pX, c);
        }
        if (lane == 5) fe_store(pY, yn);
        __syncwarp();
    }
}

// Broadcast from lane k (0..3) of this thread's quad (lanes 4i .. 4i+3) to
// the quad's four lanes; only the quad's lanes take part.
template <class F>
KB_DEV void fe_qbcast(Fe<F>& r, const Fe<F>& a, int k) {
    const unsigned qm = 0xFu << (threadIdx.x & 28);
#pragma unroll
    for (int i = 0; i < F::N; ++i) r.v[i] = __shfl_sync(qm, a.v[i], k, 4);
}

// p += q (add-2008-s) with the products spread over the four lanes of a
// quad: the 14 products fall into four dependent levels of at most four
// independent ones, so the critical path is four product latencies instead
// of fourteen.  All four lanes hold the same p and q on entry and the sum on
// return (so every branch is uniform across the quad).  For latency-bound
// reductions with spare lanes.
template <class F>
KB_DEV void xyzz_add_quad(Xyzz<F>& p, const Xyzz<F>& q) {
    if (xyzz_is_inf(q)) return;
    if (xyzz_is_inf(p)) {
        p = q;
        return;
    }
    const int ql = threadIdx.x & 3;
    Fe<F> a, b, r;
    // level 1: U1 = X1 ZZ2, U2 = X2 ZZ1, S1 = Y1 ZZZ2, S2 = Y2 ZZZ1
    a = ql == 0 ? p.X : (ql == 1 ? q.X : (ql == 2 ? p.Y : q.Y));
    b = ql == 0 ? q.ZZ : (ql == 1 ? p.ZZ : (ql == 2 ? q.ZZZ : p.ZZZ));
    fe_mul(r, a, b);
    Fe<F> U1, P, S1, R;
    fe_qbcast(U1, r, 0);
    fe_qbcast(P, r, 1);
    fe_qbcast(S1, r, 2);
    fe_qbcast(R, r, 3);
    fe_sub(P, P, U1);  // P = U2 - U1
    fe_sub(R, R, S1);  // R = S2 - S1
    if (fe_is_zero(P)) {
        if (fe_is_zero(R))
            xyzz_dbl(p, p);
        else
            xyzz_set_inf(p);
        return;
    }
    // level 2: PP = P^2, RR = R^2, ZZ1 ZZ2, ZZZ1 ZZZ2
    a = ql == 0 ? P : (ql == 1 ? R : (ql == 2 ? p.ZZ : p.ZZZ));
    b = ql == 0 ? P : (ql == 1 ? R : (ql == 2 ? q.ZZ : q.ZZZ));
    fe_mul(r, a, b);
    Fe<F> PP, RR;
    fe_qbcast(PP, r, 0);
    fe_qbcast(RR, r, 1);
    fe_qbcast(p.ZZ, r, 2);   // ZZ1 ZZ2 for now
    fe_qbcast(p.ZZZ, r, 3);  // ZZZ1 ZZZ2 for now
    // level 3: PPP = P PP, Q = U1 PP, ZZ3 = ZZ1 ZZ2 PP
    a = ql == 0 ? P : (ql == 1 ? U1 : p.ZZ);
    fe_mul(r, a, PP);
    fe_qbcast(P, r, 0);      // P <- PPP
    fe_qbcast(U1, r, 1);     // U1 <- Q
    fe_qbcast(p.ZZ, r, 2);
    fe_sub(p.X, RR, P);
    fe_sub(p.X, p.X, U1);
    fe_sub(p.X, p.X, U1);    // X3 = R^2 - PPP - 2Q
    fe_sub(U1, U1, p.X);     // Q - X3
    // level 4: R (Q - X3), S1 PPP, ZZZ3 = ZZZ1 ZZZ2 PPP
    a = ql == 0 ? R : (ql == 1 ? S1 : p.ZZZ);
    b = ql == 0 ? U1 : P;
    fe_mul(r, a, b);
    fe_qbcast(R, r, 0);
    fe_qbcast(S1, r, 1);
    fe_qbcast(p.ZZZ, r, 2);
    fe_sub(p.Y, R, S1);      // Y3 = R(Q - X3) - S1 PPP
}

// V = [k] V for a small k >= 0 by double-and-add, the doublings spread over
// the warp (xyzz_dbl_warp); every lane holds the same point and performs the
// same additions.  All 32 lanes must call it.
template <class F>
KB_DEV void xyzz_mul_small_warp(Xyzz<F>& V, uint32_t k) {
    if (k == 0) {
        xyzz_set_inf(V);
        return;
    }
    const Xyzz<F> R = V;
    for (int b = 30 - __clz(k); b >= 0; --b) {
        xyzz_dbl_warp(V);
        if ((k >> b) & 1u) xyzz_add(V, R);
    }
}

// mdbl-2008-s-1: r = 2 * (affine a).
template <class F>
KB_DEV void xyzz_mdbl(Xyzz<F>& r, const Affine<F>& a) {
    Fe<F> U, V, W, S, M, t;
    fe_dbl(U, a.y);
    fe_sqr(V, U);
    fe_mul(W, U, V);
    fe_mul(S, a.x, V);
    fe_sqr(t, a.x);
    fe_dbl(M, t);
    fe_add(M, M, t);
    fe_sqr(r.X, M);
    fe_sub(r.X, r.X, S);
    fe_sub(r.X, r.X, S);
    fe_sub(t, S, r.X);
    fe_mul(r.Y, M, t);
    fe_mul(t, W, a.y);
    fe_sub(r.Y, r.Y, t);
    r.ZZ = V;
    r.ZZZ = W;
}

// madd-2008-s: p += a, with a a finite affine point.  Temporaries are
// reused so that at most five field elements are live besides p and a.
template <class F>
KB_DEV void xyzz_add_affine(Xyzz<F>& p, const Affine<F>& a) {
    if (xyzz_is_inf(p)) {
        xyzz_from_affine(p, a);
        return;
    }
    Fe<F> P, R, t;
    fe_mul(P, a.x, p.ZZ);
    fe_sub(P, P, p.X);          // P = x2*ZZ1 - X1
    fe_mul(R, a.y, p.ZZZ);
    fe_sub(R, R, p.Y);          // R = y2*ZZZ1 - Y1
    if (fe_is_zero(P)) {
        if (fe_is_zero(R))
            xyzz_mdbl(p, a);
        else
            xyzz_set_inf(p);
        return;
    }
    Fe<F> PP, Q;
    fe_sqr(PP, P);              // PP
    fe_mul(Q, p.X, PP);         // Q = X1*PP
    fe_mul(p.ZZ, p.ZZ, PP);     // ZZ3 = ZZ1*PP
    fe_mul(PP, P, PP);          // PP <- PPP = P*PP
    fe_mul(p.ZZZ, p.ZZZ, PP);   // ZZZ3 = ZZZ1*PPP
    fe_mul(t, p.Y, PP);         // Y1*PPP
    fe_sqr(p.X, R);
    fe_sub(p.X, p.X, PP);
    fe_sub(p.X, p.X, Q);
    fe_sub(p.X, p.X, Q);        // X3 = R^2 - PPP - 2Q
    fe_sub(Q, Q, p.X);
    fe_mul(Q, R, Q);
    fe_sub(p.Y, Q, t);          // Y3 = R(Q - X3) - Y1*PPP
}

// add-2008-s: p += q, both XYZZ (either may be infinity).
template <class F>
KB_DEV void xyzz_add(Xyzz<F>& p, const Xyzz<F>& q) {
    if (xyzz_is_inf(q)) return;
    if (xyzz_is_inf(p)) {
        p = q;
        return;
    }
    Fe<F> U1, S1, P, R;
    fe_mul(U1, p.X, q.ZZ);
    fe_mul(P, q.X, p.ZZ);
    fe_sub(P, P, U1);           // P = U2 - U1
    fe_mul(S1, p.Y, q.ZZZ);
    fe_mul(R, q.Y, p.ZZZ);
    fe_sub(R, R, S1);           // R = S2 - S1
    if (fe_is_zero(P)) {
        if (fe_is_zero(R))
            xyzz_dbl(p, p);
        else
            xyzz_set_inf(p);
        return;
    }
    Fe<F> PP;
    fe_sqr(PP, P);
    fe_mul(p.ZZ, p.ZZ, q.ZZ);
    fe_mul(p.ZZ, p.ZZ, PP);     // ZZ3 = ZZ1*ZZ2*PP
    fe_mul(U1, U1, PP);         // U1 <- Q = U1*PP
    fe_mul(PP, P, PP);          // PP <- PPP = P*PP
    fe_mul(p.ZZZ, p.ZZZ, q.ZZZ);
    fe_mul(p.ZZZ, p.ZZZ, PP);   // ZZZ3 = ZZZ1*ZZZ2*PPP
    fe_mul(S1, S1, PP);         // S1*PPP
    fe_sqr(p.X, R);
    fe_sub(p.X, p.X, PP);
    fe_sub(p.X, p.X, U1);
    fe_sub(p.X, p.X, U1);       // X3 = R^2 - PPP - 2Q
    fe_sub(U1, U1, p.X);
    fe_mul(U1, R, U1);
    fe_sub(p.Y, U1, S1);        // Y3 = R(Q - X3) - S1*PPP
}

template <class F>
KB_DEV void xyzz_neg(Xyzz<F>& p) {
    fe_neg(p.Y, p.Y);
}

// Affine result (Montgomery form); returns false for infinity.
template <class F>
KB_DEV bool xyzz_to_affine(Affine<F>& a, const Xyzz<F>& p) {
    if (xyzz_is_inf(p)) return false;
    Fe<F> t, inv;
    fe_mul(t, p.ZZ, p.ZZZ);
    fe_inv(inv, t);           // 1 / (ZZ * ZZZ)
    Fe<F> izz, izzz;
    fe_mul(izz, inv, p.ZZZ);  // 1 / ZZ
    fe_mul(izzz, inv, p.ZZ);  // 1 / ZZZ
    fe_mul(a.x, p.X, izz);
    fe_mul(a.y, p.Y, izzz);
    return true;
}


// Memory helpers for XYZZ points stored as 4N consecutive words.
template <class F>
KB_DEV void xyzz_load(Xyzz<F>& p, const uint32_t* w) {  // w 16-byte aligned
    fe_load16(p.X, w);
    fe_load16(p.Y, w + F::N);
    fe_load16(p.ZZ, w + 2 * F::N);
    fe_load16(p.ZZZ, w + 3 * F::N);
}
// The same through L2 only (ld.global.cg): for records that other blocks of
// the running kernel wrote, which this SM's L1 may not see.
template <class F>
KB_DEV void xyzz_load_cg(Xyzz<F>& p, const uint32_t* w) {  // w 16-byte aligned
    const uint4* s = reinterpret_cast<const uint4*>(w);
    Fe<F>* f[4] = {&p.X, &p.Y, &p.ZZ, &p.ZZZ};
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < F::N / 4; ++k) {
            const uint4 v = __ldcg(s + c * (F::N / 4) + k);
            f[c]->v[4 * k] = v.x;
            f[c]->v[4 * k + 1] = v.y;
            f[c]->v[4 * k + 2] = v.z;
            f[c]->v[4 * k + 3] = v.w;
        }
}
template <class F>
KB_DEV void xyzz_store(uint32_t* w, const Xyzz<F>& p) {  // w 16-byte aligned
    fe_store16(w, p.X);
    fe_store16(w + F::N, p.Y);
    fe_store16(w + 2 * F::N, p.ZZ);
    fe_store16(w + 3 * F::N, p.ZZZ);
}

// An XYZZ point held in shared memory, word-major over a block of STRIDE
// threads: coordinate f (0 = X, 1 = Y, 2 = ZZ, 3 = ZZZ), word k of this
// thread at base[(f * N + k) * STRIDE].  Consecutive threads hit consecutive
// banks.  An accumulator kept here rather than in registers leaves only the
// temporaries of the formula in registers, which raises the resident warps
// per SM of the latency-bound addition kernels.
template <class F, int STRIDE>
struct SmXyzz {
    uint32_t* base;  // shared array + threadIdx.x
    KB_DEV void get(int f, Fe<F>& r) const {
#pragma unroll
        for (int k = 0; k < F::N; ++k) r.v[k] = base[(f * F::N + k) * STRIDE];
    }
    KB_DEV void put(int f, const Fe<F>& r) const {
#pragma unroll
        for (int k = 0; k < F::N; ++k) base[(f * F::N + k) * STRIDE] = r.v[k];
    }
    KB_DEV bool is_inf() const {
        uint32_t o = 0;
#pragma unroll
        for (int k = 0; k < F::N; ++k) o |= base[(2 * F::N + k) * STRIDE];
        return o == 0;
    }
    KB_DEV void set_inf() const {
#pragma unroll
        for (int k = 0; k < 4 * F::N; ++k) base[k * STRIDE] = 0;
    }
    KB_DEV void to_global(uint32_t* w) const {  // w 16-byte aligned
        uint4* d = reinterpret_cast<uint4*>(w);
#pragma unroll
        for (int k = 0; k < F::N; ++k)
            d[k] = make_uint4(base[(4 * k) * STRIDE], base[(4 * k + 1) * STRIDE],
                              base[(4 * k + 2) * STRIDE], base[(4 * k + 3) * STRIDE]);
    }
};

// Read-only view of an XYZZ point stored as 4N consecutive words in global
// memory, with the accessors of SmXyzz.
template <class F>
struct GXyzz {
    const uint32_t* w;
    KB_DEV void get(int f, Fe<F>& r) const { fe_load16(r, w + f * F::N); }  // w 16-byte aligned
    KB_DEV bool is_inf() const {
        uint32_t o = 0;
#pragma unroll
        for (int k = 0; k < F::N; ++k) o |= w[2 * F::N + k];
        return o == 0;
    }
};

template <class F, int S, class Q>
KB_DEV void xyzz_copy(const SmXyzz<F, S>& p, const Q& q) {
    Fe<F> t;
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
        q.get(f, t);
        p.put(f, t);
    }
}

// dbl-2008-s-1 in place on a shared-memory point.
template <class F, int S>
KB_DEV void xyzz_dbl(const SmXyzz<F, S>& p) {
    Fe<F> U, V, W, t;
    p.get(1, t);
    fe_dbl(U, t);
    fe_sqr(V, U);
    fe_mul(W, U, V);
    p.get(2, t);
    fe_mul(t, V, t);
    p.put(2, t);                // ZZ3 = V*ZZ1
    p.get(0, t);
    fe_mul(U, t, V);            // U <- S = X1*V
    p.get(3, t);
    fe_mul(t, W, t);
    p.put(3, t);                // ZZZ3 = W*ZZZ1
    p.get(1, t);
    fe_mul(W, W, t);            // W <- W*Y1
    p.get(0, t);
    fe_sqr(V, t);
    fe_dbl(t, V);
    fe_add(V, V, t);            // V <- M = 3 X1^2
    fe_sqr(t, V);
    fe_sub(t, t, U);
    fe_sub(t, t, U);            // X3 = M^2 - 2S
    p.put(0, t);
    fe_sub(U, U, t);
    fe_mul(U, V, U);
    fe_sub(U, U, W);            // Y3 = M(S - X3) - W*Y1
    p.put(1, U);
}

// add-2008-s on a shared-memory accumulator: p += q, q an SmXyzz or GXyzz
// (either may be infinity; q must not alias p).  One out-of-line copy per
// kernel; its first four products, two independent pairs, are inlined so
// each pair's instruction streams interleave (stage-1 reduction at 2^22:
// 1.43 -> 1.36 ms, at 2^18: 0.99 -> 0.84 ms).
template <class F, int S, class Q>
__device__ __noinline__ void xyzz_add(const SmXyzz<F, S> p, const Q q) {
    if (q.is_inf()) return;
    if (p.is_inf()) {
        xyzz_copy(p, q);
        return;
    }
    Fe<F> U1, S1, P, R, t;
    {
        Fe<F> t2;
        q.get(2, t);
        p.get(0, U1);
        p.get(2, t2);
        q.get(0, P);
        fe_mul_inl(U1, U1, t);  // U1 = X1*ZZ2
        fe_mul_inl(P, P, t2);
        fe_sub(P, P, U1);       // P = X2*ZZ1 - U1
        q.get(3, t);
        p.get(1, S1);
        p.get(3, t2);
        q.get(1, R);
        fe_mul_inl(S1, S1, t);  // S1 = Y1*ZZZ2
        fe_mul_inl(R, R, t2);
        fe_sub(R, R, S1);       // R = Y2*ZZZ1 - S1
    }
    if (fe_is_zero(P)) {
        if (fe_is_zero(R))
            xyzz_dbl(p);
        else
            p.set_inf();
        return;
    }
    fe_sqr(t, P);               // t = PP
    fe_mul(U1, U1, t);          // U1 <- Q = U1*PP
    fe_mul(P, P, t);            // P <- PPP
    {
        Fe<F> z;
        p.get(2, z);
        fe_mul(t, t, z);
        q.get(2, z);
        fe_mul(t, t, z);
        p.put(2, t);            // ZZ3 = ZZ1*ZZ2*PP
        p.get(3, t);
        q.get(3, z);
        fe_mul(t, t, z);
        fe_mul(t, t, P);
        p.put(3, t);            // ZZZ3 = ZZZ1*ZZZ2*PPP
    }
    fe_mul(S1, S1, P);          // S1*PPP
    fe_sqr(t, R);
    fe_sub(t, t, P);
    fe_sub(t, t, U1);
    fe_sub(t, t, U1);           // X3 = R^2 - PPP - 2Q
    p.put(0, t);
    fe_sub(U1, U1, t);
    fe_mul(U1, R, U1);
    fe_sub(U1, U1, S1);         // Y3 = R(Q - X3) - S1*PPP
    p.put(1, U1);
}

// p += q (add-2008-s) for points in shared memory, the products spread over
// the four lanes of a quad in four dependent levels as in xyzz_add_quad, but
// with every operand and product passing through shared memory (t0, t1: two
// scratch points of the quad, not aliasing p or q), so no lane holds a whole
// point: for kernels whose register budget is tight, where the quad's latency
// (four product latencies instead of fourteen) matters.  All four lanes of
// the quad call it with the same arguments; q must not alias p.
template <class F, int S>
__device__ __noinline__ void xyzz_add_quad_sm(const SmXyzz<F, S> p, const SmXyzz<F, S> q,
                                              const SmXyzz<F, S> t0, const SmXyzz<F, S> t1) {
    const int ql = threadIdx.x & 3;
    const unsigned qm = 0xFu << (threadIdx.x & 28);
    if (q.is_inf()) return;
    if (p.is_inf()) {
        Fe<F> c;
        q.get(ql, c);
        p.put(ql, c);
        __syncwarp(qm);
        return;
    }
    Fe<F> a, b, r;
    // level 1: U1 = X1 ZZ2 (0), U2 = X2 ZZ1 (1), S1 = Y1 ZZZ2 (2), S2 = Y2 ZZZ1 (3) -> t0
    ((ql & 1) ? q : p).get(ql < 2 ? 0 : 1, a);
    ((ql & 1) ? p : q).get(ql < 2 ? 2 : 3, b);
    fe_mul(r, a, b);
    t0.put(ql, r);
    __syncwarp(qm);
    Fe<F> P, R;
    t0.get(0, a);
    t0.get(1, P);
    fe_sub(P, P, a);  // P = U2 - U1
    t0.get(2, a);
    t0.get(3, R);
    fe_sub(R, R, a);  // R = S2 - S1
    if (fe_is_zero(P)) {
        __syncwarp(qm);
        if (ql == 0) {
            if (fe_is_zero(R))
                xyzz_dbl(p);
            else
                p.set_inf();
        }
        __syncwarp(qm);
        return;
    }
    // level 2: PP (0), RR (1), ZZ1 ZZ2 (2), ZZZ1 ZZZ2 (3) -> t1
    if (ql >= 2) {
        p.get(ql, a);
        q.get(ql, b);
    } else {
        a = ql ? R : P;
        b = a;
    }
    fe_mul(r, a, b);
    t1.put(ql, r);
    __syncwarp(qm);
    // level 3: PPP = P PP (0) -> t0[1], Q = U1 PP (1) -> t0[3], ZZ3 = ZZ1 ZZ2 PP (2) -> p.ZZ
    t1.get(0, b);
    if (ql == 1)
        t0.get(0, a);
    else if (ql == 2)
        t1.get(2, a);
    else
        a = P;
    fe_mul(r, a, b);
    if (ql == 0) t0.put(1, r);
    if (ql == 1) t0.put(3, r);
    if (ql == 2) p.put(2, r);
    __syncwarp(qm);
    // X3 = RR - PPP - 2Q
    Fe<F> X3, QmX;
    t1.get(1, X3);
    t0.get(1, a);
    fe_sub(X3, X3, a);
    t0.get(3, QmX);
    fe_sub(X3, X3, QmX);
    fe_sub(X3, X3, QmX);
    fe_sub(QmX, QmX, X3);
    // level 4: R (Q - X3) (0), S1 PPP (1) -> t1[0], ZZZ3 = ZZZ1 ZZZ2 PPP (2) -> p.ZZZ
    if (ql == 0) {
        a = R;
        b = QmX;
    } else {
        t0.get(1, b);
        if (ql == 1)
            t0.get(2, a);
        else
            t1.get(3, a);
    }
    fe_mul(r, a, b);
    if (ql == 1) t1.put(0, r);
    if (ql == 2) p.put(3, r);
    __syncwarp(qm);
    if (ql == 0) {
        t1.get(0, a);
        fe_sub(r, r, a);  // Y3 = R (Q - X3) - S1 PPP
        p.put(0, X3);
        p.put(1, r);
    }
    __syncwarp(qm);
}

// mdbl-2008-s-1 into a shared-memory point: p = 2 * (affine a).
template <class F, int S>
KB_DEV void xyzz_mdbl_sm(const SmXyzz<F, S>& p, const Affine<F>& a) {
    Fe<F> U, V, W, t;
    fe_dbl(U, a.y);
    fe_sqr(V, U);
    fe_mul(W, U, V);
    p.put(3, W);                // ZZZ3 = W
    fe_mul(U, a.x, V);          // U <- S = x*V
    p.put(2, V);                // ZZ3 = V
    fe_sqr(t, a.x);
    fe_dbl(V, t);
    fe_add(V, V, t);            // V <- M = 3x^2
    fe_sqr(t, V);
    fe_sub(t, t, U);
    fe_sub(t, t, U);            // X3 = M^2 - 2S
    p.put(0, t);
    fe_sub(U, U, t);
    fe_mul(U, V, U);            // M(S - X3)
    fe_mul(W, W, a.y);
    fe_sub(U, U, W);            // Y3 = M(S - X3) - W*y
    p.put(1, U);
}

// madd-2008-s on a shared-memory accumulator: p += a, a finite affine
// point.  At most five field elements are live in registers besides a.
template <class F, int S>
KB_DEV void xyzz_add_affine(const SmXyzz<F, S>& p, const Affine<F>& a) {
    Fe<F> P, R, t;
    p.get(2, t);
    if (fe_is_zero(t)) {
        p.put(0, a.x);
        p.put(1, a.y);
        fe_one(t);
        p.put(2, t);
        p.put(3, t);
        return;
    }
    {
        // the two independent products inlined so they interleave
        // (accumulation at 2^22: 2.14 -> 2.02 ms)
        Fe<F> t3;
        p.get(3, t3);
        fe_mul_inl(P, a.x, t);
        fe_mul_inl(R, a.y, t3);
    }
    p.get(0, t);
    fe_sub(P, P, t);            // P = x2*ZZ1 - X1
    p.get(1, t);
    fe_sub(R, R, t);            // R = y2*ZZZ1 - Y1
    if (fe_is_zero(P)) {
        if (fe_is_zero(R))
            xyzz_mdbl_sm(p, a);
        else
            p.set_inf();
        return;
    }
    Fe<F> PP, Q;
    fe_sqr(PP, P);              // PP
    p.get(0, t);
    fe_mul(Q, t, PP);           // Q = X1*PP
    p.get(2, t);
    fe_mul(t, t, PP);
    p.put(2, t);                // ZZ3 = ZZ1*PP
    fe_mul(PP, P, PP);          // PP <- PPP
    p.get(3, t);
    fe_mul(t, t, PP);
    p.put(3, t);                // ZZZ3 = ZZZ1*PPP
    p.get(1, t);
    fe_mul(P, t, PP);           // P <- Y1*PPP
    fe_sqr(t, R);
    fe_sub(t, t, PP);
    fe_sub(t, t, Q);
    fe_sub(t, t, Q);            // X3 = R^2 - PPP - 2Q
    p.put(0, t);
    fe_sub(Q, Q, t);
    fe_mul(Q, R, Q);
    fe_sub(Q, Q, P);            // Y3 = R(Q - X3) - Y1*PPP
    p.put(1, Q);
}

// Affine table entry (2N words) -> Affine<F>; the infinity flag is masked.
template <class F>
KB_DEV void aff_load(Affine<F>& a, const uint32_t* w) {
    fe_load(a.x, w);
    a.x.v[F::N - 1] &= ~INF_FLAG;
    fe_load(a.y, w + F::N);
}

// Wire (big-endian x || y, all-zero = infinity) -> internal table entry.
template <class C>
KB_DEV void wire_to_table(uint32_t* dst, const uint8_t* wire) {
    using F = typename C::F;
    uint32_t any = 0;
    for (int i = 0; i < C::WIRE; ++i) any |= wire[i];
    if (!any) {
        for (int i = 0; i < 2 * F::N; ++i) dst[i] = 0;
        dst[F::N - 1] = INF_FLAG;
        return;
    }
    Fe<F> x, y;
    fe_from_be_bytes(x, wire);
    fe_from_be_bytes(y, wire + F::BYTES);
    fe_to_mont(x, x);
    fe_to_mont(y, y);
    fe_store(dst, x);
    fe_store(dst + F::N, y);
}

// XYZZ -> wire bytes (canonical affine big-endian, zeros for infinity).
template <class C>
KB_DEV void xyzz_to_wire(uint8_t* wire, const Xyzz<typename C::F>& p) {
    using F = typename C::F;
    Affine<F> a;
    if (!xyzz_to_affine(a, p)) {
        for (int i = 0; i < C::WIRE; ++i) wire[i] = 0;
        return;
    }
    Fe<F> x, y;
    fe_from_mont(x, a.x);
    fe_from_mont(y, a.y);
    fe_to_be_bytes(wire, x);
    fe_to_be_bytes(wire + F::BYTES, y);
}

}  // namespace kb200
