"""Input builders for the EIP-2537 G1 MSM tests (test infrastructure):
160-byte entries x[64] || y[64] || c[32], big endian, from points the oracle
makes, plus the invalid encodings the precompile must reject."""
from __future__ import annotations

import random

import _oracle as O

P = O.FP[2]
R = O.FR[2]


def pad64(v: int) -> bytes:
    return v.to_bytes(64, "big")


def entry(point96: bytes, scalar: int) -> bytes:
    x = int.from_bytes(point96[:48], "big")
    y = int.from_bytes(point96[48:], "big")
    return pad64(x) + pad64(y) + scalar.to_bytes(32, "big")


def g1_point(k: int) -> bytes:
    return O.g1_mul_gen(2, k)


def curve_point_not_in_g1(rng: random.Random) -> bytes:
    """A random point of E(Fp): its order has a cofactor part, so it lies
    outside G1 (probability of landing in G1 ~ 2^-126)."""
    while True:
        x = rng.randrange(P)
        t = (x * x * x + 4) % P
        y = pow(t, (P + 1) // 4, P)
        if y * y % P == t:
            return x.to_bytes(48, "big") + y.to_bytes(48, "big")


def torsion_point(rng: random.Random) -> bytes:
    """[r]Q for a random curve point Q: a point of cofactor order."""
    while True:
        out = O.g1_mul(2, curve_point_not_in_g1(rng), R)
        if any(out):
            return out


def valid_input(rng: random.Random, n: int, inf_every: int = 0, full_scalars: bool = True):
    ents, pts, scs = [], [], []
    for i in range(n):
        if inf_every and i % inf_every == inf_every - 1:
            ents.append(bytes(128) + rng.getrandbits(256).to_bytes(32, "big"))
            continue
        p = g1_point(rng.randrange(1, R))
        s = rng.getrandbits(256) if full_scalars else rng.randrange(R)
        ents.append(entry(p, s))
        pts.append(p)
        scs.append(s % R)
    return b"".join(ents), pts, scs


def expected(pts, scs) -> bytes:
    """rx || ry from the oracle's G1 MSM of the finite points."""
    if not pts:
        return bytes(128)
    out = O.msm(2, b"".join(s.to_bytes(32, "little") for s in scs), b"".join(pts), len(pts))
    return bytes(16) + out[:48] + bytes(16) + out[48:]
