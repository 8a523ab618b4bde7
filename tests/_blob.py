"""Helpers for the EIP-4844 blob tests (test infrastructure): seeded blobs,
domain points, and the monomial / Lagrange setups for a test tau."""
from __future__ import annotations

import random
from functools import lru_cache

import _oracle as O

R = O.FR[2]
N = 4096
W = pow(7, (R - 1) // N, R)


def brp(i: int, bits: int = 12) -> int:
    return int(format(i, f"0{bits}b")[::-1], 2)


def domain_point(i: int) -> int:
    """w^brp(i): the point blob element i is the value at."""
    return pow(W, brp(i), R)


def rand_blob(seed: int) -> bytes:
    rng = random.Random(seed)
    return b"".join(rng.randrange(R).to_bytes(32, "big") for _ in range(N))


TAU = 0x2F1C8A6B3D5E7F90123456789ABCDEF0FEDCBA9876543210A1B2C3D4E5F60718 % R


@lru_cache(maxsize=1)
def monomial_srs() -> bytes:
    """[tau^i]G1, i < 4096, for the oracle (96 B BE each)."""
    powers = O.fr_powers(2, TAU.to_bytes(32, "little"), N)
    return b"".join(O.g1_mul_gen(2, int.from_bytes(powers[32 * i:32 * i + 32], "little"))
                    for i in range(N))


def lagrange_compressed() -> bytes:
    """The setup's Lagrange points [L_j(tau)]G1 in natural order j,
    48-byte compressed: the layout of a trusted-setup file."""
    tn = pow(TAU, N, R) - 1
    ninv = pow(N, R - 2, R)
    out = []
    for j in range(N):
        wj = pow(W, j, R)
        lj = wj * tn * ninv * pow((TAU - wj) % R, R - 2, R) % R
        out.append(O.compress(O.g1_mul_gen(2, lj)))
    return b"".join(out)
