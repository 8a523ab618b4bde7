"""CPU restatement of the G1 membership test the device runs for EIP-2537
inputs and blob setups (crypto_b200/csrc/g1check.cuh): sigma(P) = -[u^2]P
evaluated as two [|u|] double-and-add chains in Jacobian coordinates, with
the same formulas and the same edge-case branches (infinity, equal and
opposite operands) as the device code.  Checked against the definition
([r]P = O) on G1 points, random curve points and torsion points of every
prime-power order dividing the cofactor, plus torsion + G1 sums.  The device
path itself is compared with the oracle in test_eip2537_gpu.py."""
from __future__ import annotations

import random

import _oracle as O

P = O.FP[2]
R = O.FR[2]
U_ABS = 0xD201000000010000
H1 = 0x396C8C005555E1568C00AAAB0000AAAB  # G1 cofactor
# primitive cube root of unity with sigma(x, y) = (BETA x, y) = [-u^2] on G1
BETA = 0x5F19672FDF76CE51BA69C6076A0F77EADDB3A93BE6F89688DE17D813620A00022E01FFFFFFFEFFFE
GEN = (0x17F1D3A73197D7942695638C4FA9AC0FC3688C4F9774B905A14E3A3F171BAC586C55E83FF97A1AEFFB3AF00ADB22C6BB,
       0x08B3F481E3AAA0F1A09E30ED741D8AE4FCF5E095D5D00AF600DB18CB2C04B3EDD03CC744A2888AE40CAA232946C5E7E1)
# prime-power factors of the cofactor: 3, 11^2, 10177^2, 859267^2, 52437899^2
COFACTOR_PARTS = (3, 11 ** 2, 10177 ** 2, 859267 ** 2, 52437899 ** 2)


def _inv(a):
    return pow(a, P - 2, P)


def aff_add(p1, p2):
    if p1 is None:
        return p2
    if p2 is None:
        return p1
    (x1, y1), (x2, y2) = p1, p2
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        lam = 3 * x1 * x1 * _inv(2 * y1) % P
    else:
        lam = (y2 - y1) * _inv(x2 - x1) % P
    x3 = (lam * lam - x1 - x2) % P
    return x3, (lam * (x1 - x3) - y1) % P


def aff_mul(k, p):
    acc = None
    while k:
        if k & 1:
            acc = aff_add(acc, p)
        p = aff_add(p, p)
        k >>= 1
    return acc


# ---- the device's formula sequence (g1check.cuh) ---------------------------

def j_dbl(p):
    """dbl-2009-l, a = 0."""
    X, Y, Z = p
    A = X * X % P
    B = Y * Y % P
    C = B * B % P
    D = 2 * ((X + B) * (X + B) - A - C) % P
    E = 3 * A % P
    X3 = (E * E - 2 * D) % P
    return X3, (E * (D - X3) - 8 * C) % P, 2 * Y * Z % P


def j_madd(p, a):
    """madd-2007-bl: p += a, a finite affine."""
    X1, Y1, Z1 = p
    if Z1 == 0:
        return a[0], a[1], 1
    Z1Z1 = Z1 * Z1 % P
    H = (a[0] * Z1Z1 - X1) % P
    r = 2 * (a[1] * Z1 * Z1Z1 - Y1) % P
    if H == 0:
        return j_dbl(p) if r == 0 else (1, 1, 0)
    HH = H * H % P
    I = 4 * HH % P
    J = H * I % P
    V = X1 * I % P
    X3 = (r * r - J - 2 * V) % P
    return X3, (r * (V - X3) - 2 * Y1 * J) % P, ((Z1 + H) ** 2 - Z1Z1 - HH) % P


def j_add_cached(p, q, qzz, qzzz):
    """add-2007-bl: p += q, q finite with qzz = Zq^2, qzzz = Zq^3."""
    X1, Y1, Z1 = p
    if Z1 == 0:
        return q
    X2, Y2, Z2 = q
    Z1Z1 = Z1 * Z1 % P
    U1 = X1 * qzz % P
    S1 = Y1 * qzzz % P
    H = (X2 * Z1Z1 - U1) % P
    r = 2 * (Y2 * Z1 * Z1Z1 - S1) % P
    if H == 0:
        return j_dbl(p) if r == 0 else (1, 1, 0)
    I = (2 * H) ** 2 % P
    J = H * I % P
    V = U1 * I % P
    X3 = (r * r - J - 2 * V) % P
    return X3, (r * (V - X3) - 2 * S1 * J) % P, ((Z1 + Z2) ** 2 - Z1Z1 - qzz) * H % P


def in_g1_device_formulas(a) -> bool:
    q = (a[0], a[1], 1)
    for b in range(62, -1, -1):
        q = j_dbl(q)
        if (U_ABS >> b) & 1:
            q = j_madd(q, a)
    if q[2] == 0:
        return False
    q1, qzz = q, q[2] * q[2] % P
    qzzz = qzz * q[2] % P
    for b in range(62, -1, -1):
        q = j_dbl(q)
        if (U_ABS >> b) & 1:
            q = j_add_cached(q, q1, qzz, qzzz)
    X, Y, Z = q
    if Z == 0:
        return False
    zz = Z * Z % P
    return BETA * a[0] * zz % P == X and (P - a[1]) * zz * Z % P == Y


def in_g1_definition(a) -> bool:
    return aff_mul(R, a) is None


def random_curve_point(rng):
    while True:
        x = rng.randrange(P)
        t = (x ** 3 + 4) % P
        y = pow(t, (P + 1) // 4, P)
        if y * y % P == t:
            return x, y


def test_cofactor_parts():
    prod = 1
    for f in COFACTOR_PARTS:
        prod *= f
    assert prod == H1


def test_beta_is_minus_u_squared_on_g1():
    assert aff_mul(U_ABS * U_ABS % R, GEN) == (BETA * GEN[0] % P, (P - GEN[1]) % P)


def test_g1_points_accepted():
    rng = random.Random(1)
    for _ in range(4):
        g = aff_mul(rng.randrange(1, R), GEN)
        assert in_g1_device_formulas(g) and in_g1_definition(g)


def test_random_curve_points_rejected():
    rng = random.Random(2)
    for _ in range(4):
        q = random_curve_point(rng)
        assert not in_g1_device_formulas(q) and not in_g1_definition(q)


def test_torsion_points_rejected():
    rng = random.Random(3)
    for f in COFACTOR_PARTS:
        T = None
        while T is None:
            T = aff_mul(H1 // f * R, random_curve_point(rng))  # order divides f
        assert not in_g1_device_formulas(T) and not in_g1_definition(T), f
        S = aff_add(T, aff_mul(rng.randrange(1, R), GEN))  # torsion + G1
        assert not in_g1_device_formulas(S) and not in_g1_definition(S), f
