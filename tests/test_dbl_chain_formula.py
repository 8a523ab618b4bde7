"""The two-level doubling chain of the window weighting (xyzz_dbl_chain_warp_sm in
crypto_b200/csrc/curve.cuh) restated over Python integers: k doublings carried with X^2,
3X^3 and 2Y^2 must give the same XYZZ coordinates as k doublings by dbl-2008-s-1 (the
formula of xyzz_dbl), for any inputs, since both are the same polynomials.  The device
chain itself is covered by the MSM parity tests (every window weight passes through it)."""
import random

import pytest

P_BLS = int(
    "1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab",
    16)
P_BN = int("30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47", 16)


def dbl_2008_s_1(P, p):
    X, Y, ZZ, ZZZ = P
    U = 2 * Y % p
    V = U * U % p
    W = U * V % p
    S = X * V % p
    M = 3 * X * X % p
    X3 = (M * M - 2 * S) % p
    Y3 = (M * (S - X3) - W * Y) % p
    return X3, Y3, V * ZZ % p, W * ZZZ % p


def chain(P, k, p):
    X, Y, ZZ, ZZZ = P
    X2 = X * X % p
    Y2 = 2 * Y * Y % p  # 2Y^2
    X3 = 3 * X * X2 % p  # 3X^3
    for _ in range(k):
        t = (X3 - Y2) % p
        u = (3 * t - Y2) % p  # 9X^3 - 8Y^2
        # level 1
        Xn, U2, VU, T, Y3, ZZ = X * u % p, u * u % p, X3 * u % p, Y2 * t % p, Y * Y2 % p, 2 * (ZZ * Y2) % p
        yn = (2 * T - VU) % p
        # level 2
        X2, X3, Y2, ZZZ = X2 * U2 % p, VU * U2 % p, 2 * yn * yn % p, 4 * (Y3 * ZZZ) % p
        X, Y = Xn, yn
    return X, Y, ZZ, ZZZ


@pytest.mark.parametrize("p", [P_BLS, P_BN], ids=["bls12_381", "bn254"])
def test_chain_matches_repeated_doubling(p):
    rng = random.Random(7)
    for _ in range(25):
        P = tuple(rng.randrange(p) for _ in range(4))
        k = rng.randrange(0, 48)
        Q = P
        for _ in range(k):
            Q = dbl_2008_s_1(Q, p)
        assert chain(P, k, p) == Q
