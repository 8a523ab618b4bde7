"""CPU checks of the GLV constants the MSM kernels embed (msm_kernels.cuh,
curve.cuh, msm.cu), read from the source files: the endomorphism pairs
(beta, lambda) act as phi(x, y) = (beta x, y) = [lambda](x, y) on the
generator; the BN254 lattice basis, its rounding constants and the device's
integer split formula give k1 + k2 lambda = k (mod r) with both halves
inside the bound the window planner assumes, at random scalars and at the
rounding boundaries; the BLS12-381 split k = k1 + k2 lambda by division
stays below its bound too."""
from __future__ import annotations

import random
import re
from pathlib import Path

import _oracle as O

SRC = Path(__file__).resolve().parents[1] / "crypto_b200" / "csrc"


def const_words(name: str) -> int:
    """Integer value of a little-endian uint32_t constant array in the sources."""
    for f in SRC.glob("*.cu*"):
        m = re.search(r"\b%s\[\d+\]\s*=\s*\{([^}]*)\}" % re.escape(name), f.read_text())
        if m:
            words = [int(w, 16) for w in re.findall(r"0x[0-9a-fA-F]+", m.group(1))]
            return sum(w << (32 * i) for i, w in enumerate(words))
    raise KeyError(name)


def glv_bound(curve: int) -> int:
    text = (SRC / "msm.cu").read_text()
    body = text[text.index("static unsigned __int128 glv_bound"):]
    hexes = [int(h, 16) for h in re.findall(r"0x([0-9a-fA-F]+)ull", body)[:4]]
    bls = (hexes[0] << 64) | hexes[1]
    bn = (hexes[2] << 64) | hexes[3]
    return bls if curve == 2 else bn


def from_mont(v: int, p: int, bits: int) -> int:
    return v * pow(2, -bits, p) % p


def test_endomorphism_pairs_match_on_generator():
    for curve, beta_name, bits, lam in (
            (2, "kGlvBeta2Mont", 384, const_words("kGlvLambda")),
            (1, "kBnGlvBetaMont", 256, 0xB3C4D79D41A917585BFC41088D8DAAA78B17EA66B99C90DD)):
        p, r = O.FP[curve], O.FR[curve]
        beta = from_mont(const_words(beta_name), p, bits)
        assert pow(beta, 3, p) == 1 and beta != 1
        assert (lam * lam + lam + 1) % r == 0
        g = O.g1_mul_gen(curve, 1)
        w = len(g) // 2
        x = int.from_bytes(g[:w], "big")
        phi_g = (beta * x % p).to_bytes(w, "big") + g[w:]
        assert O.g1_mul_gen(curve, lam) == phi_g


def test_bn254_split_exact_and_bounded():
    r = O.FR[1]
    lam = 0xB3C4D79D41A917585BFC41088D8DAAA78B17EA66B99C90DD
    a1, b1 = const_words("kBnGlvA1"), const_words("kBnGlvB1")
    a2, b2 = const_words("kBnGlvA2"), const_words("kBnGlvB2")
    g1, g2 = const_words("kBnGlvG1"), const_words("kBnGlvG2")
    # basis v1 = (a1, -b1), v2 = (a2, b2) of {(x, y): x + y lambda = 0 mod r}, det r
    assert (a1 - b1 * lam) % r == 0 and (a2 + b2 * lam) % r == 0
    assert a1 * b2 + b1 * a2 == r
    assert g2 == (2**384 * b2 + r // 2) // r and g1 == (2**384 * b1 + r // 2) // r
    assert const_words("kBnR256ModR") == 2**256 % r
    bound = glv_bound(1)
    assert bound.bit_length() == 126

    def split(k):  # the device formula (msm_kernels.cuh glv_split_bn)
        ca = (k * g2 + 2**383) >> 384
        cb = (k * g1 + 2**383) >> 384
        return k - ca * a1 - cb * a2, ca * b1 - cb * b2

    rng = random.Random(7)
    ks = [0, 1, 2, r - 1, r - 2, lam, lam + 1, r // 2] + [rng.randrange(r) for _ in range(20000)]
    for b in (b1, b2):
        for _ in range(2000):
            c = (2 * rng.randrange(1, b) + 1) * r // (2 * b)
            ks += [c % r, (c + 1) % r, (c - 1) % r]
    for k in ks:
        k1, k2 = split(k)
        assert (k1 + k2 * lam - k) % r == 0
        assert abs(k1) < bound and abs(k2) < bound


def test_bls12_381_split_bounded():
    r = O.FR[2]
    lam = const_words("kGlvLambda")
    assert lam * lam + lam + 1 == r
    assert const_words("kGlvMu") == 2**384 // lam
    assert const_words("kR256ModR") == 2**256 % r
    bound = glv_bound(2)
    assert bound == max(lam - 1, (r - 1) // lam)
    rng = random.Random(3)
    for k in [0, 1, r - 1, lam, lam - 1] + [rng.randrange(r) for _ in range(5000)]:
        k1, k2 = k % lam, k // lam
        assert k1 <= bound and k2 <= bound
