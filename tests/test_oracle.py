"""CPU checks of the oracle itself (no GPU): it must reproduce the reference's
golden vectors and the reference's own CPU MSM before any GPU result is
compared against it."""
from __future__ import annotations

import gzip
import json
import random
from pathlib import Path

import pytest

import _oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden.json.gz"


@pytest.fixture(scope="module")
def golden():
    with gzip.open(GOLDEN, "rt") as f:
        return json.load(f)


def test_golden_msm(golden):
    for c in golden["msm"]:
        got = O.msm(c["curve"], bytes.fromhex(c["scalars"]), bytes.fromhex(c["points"]), c["n"])
        assert got.hex() == c["expected"], (c["curve"], c["n"], c["mode"])


def test_golden_ntt(golden):
    for c in golden["ntt"]:
        got = O.ntt(c["curve"], bytes.fromhex(c["input"]), bool(c["inverse"]), bool(c["coset"]))
        assert got.hex() == c["expected"], (c["curve"], c["n"], c["inverse"], c["coset"])


def test_golden_kzg(golden):
    for c in golden["kzg"]:
        got = O.kzg_commit(bytes.fromhex(c["evals"]), bytes.fromhex(c["srs"]))
        assert got.hex() == c["commit"]


def test_compressed_generator_vector():
    # kzg/test/kzg_test.cpp:64-81: compressed G1 generator = x with 0x80 only;
    # :38-42: infinity = 0xC0 followed by zeros.
    g = O.g1_mul_gen(2, 1)
    c = O.compress(g)
    x = bytes.fromhex("17F1D3A73197D7942695638C4FA9AC0FC3688C4F9774B905A14E3A3F171BAC58"
                      "6C55E83FF97A1AEFFB3AF00ADB22C6BB")
    assert c == bytes([x[0] | 0x80]) + x[1:]
    assert O.compress(bytes(96)) == b"\xc0" + bytes(47)
    # -G has the larger y, so the sign bit is set.
    neg = O.g1_mul_gen(2, O.FR[2] - 1)
    assert O.compress(neg)[0] == (x[0] | 0xA0)


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("curve", [1, 2])
def test_oracle_matches_reference_random(curve):
    rng = random.Random(7 + curve)
    for n in (3, 33, 130):
        pts = b"".join(O.g1_mul_gen(curve, rng.getrandbits(250)) for _ in range(n))
        scs = b"".join(rng.getrandbits(256).to_bytes(32, "little") for _ in range(n))
        assert O.msm(curve, scs, pts, n) == O.ref_msm(curve, scs, pts, n)
        # The composed parallel reference equals the plain one by the group
        # law -- for scalars below 2^255 only, since the reference's dropped
        # top carry depends on the slice size through its window choice.
        can = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
        assert O.ref_msm(curve, can, pts, n, threads=4) == O.ref_msm(curve, can, pts, n)


@pytest.mark.parametrize("curve", [1, 2])
def test_msm_matches_naive_for_canonical_scalars(curve):
    rng = random.Random(11)
    n = 40
    pts = b"".join(O.g1_mul_gen(curve, rng.getrandbits(250)) for _ in range(n))
    scs = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
    assert O.msm(curve, scs, pts, n) == O.msm_naive(curve, scs, pts, n)


@pytest.mark.parametrize("curve", [1, 2])
def test_ntt_matches_dft_and_round_trips(curve):
    rng = random.Random(3)
    for logn in range(0, 8):
        n = 1 << logn
        x = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
        for coset in (False, True):
            y = O.ntt(curve, x, False, coset)
            assert y == O.dft(curve, x, False, coset)
            assert O.ntt(curve, y, True, coset) == x


@pytest.mark.parametrize("curve", [1, 2])
def test_ntt_is_polynomial_evaluation(curve):
    """Forward NTT of coefficients = evaluations at w^k (Horner), and w has order n."""
    r = O.FR[curve]
    rng = random.Random(5)
    n = 32
    coeffs = [rng.randrange(r) for _ in range(n)]
    y = O.ntt(curve, b"".join(c.to_bytes(32, "little") for c in coeffs))
    import ctypes
    buf = ctypes.create_string_buffer(32)
    assert O.orc().orc_root_of_unity(curve, n, buf) == 0
    w = int.from_bytes(buf.raw, "little")
    assert pow(w, n, r) == 1 and pow(w, n // 2, r) != 1
    for k in (0, 1, 5, n - 1):
        x = pow(w, k, r)
        acc = 0
        for c in reversed(coeffs):
            acc = (acc * x + c) % r
        assert int.from_bytes(y[32 * k:32 * k + 32], "little") == acc


def test_root_generators_are_nonresidues():
    # g = 7 (BLS12-381 Fr) and g = 5 (BN254 Fr) generate the full 2-adic subgroup.
    for curve, g in ((2, 7), (1, 5)):
        r = O.FR[curve]
        assert pow(g, (r - 1) // 2, r) == r - 1


def test_points_on_curve():
    for curve in (1, 2):
        assert O.on_curve(curve, O.g1_mul_gen(curve, 12345))
        assert O.on_curve(curve, bytes(O.PB[curve]))


@pytest.mark.parametrize("curve", [1, 2])
def test_cpu_input_generators_match_library(curve):
    """The CPU-only legs (reference arm, golden script) rebuild the workload
    with the oracle's restated generators: the same scalar streams as the
    library's kb200_gen_scalars, and fixed-base points equal to the
    double-and-add k * G of the oracle."""
    import crypto_b200 as kb
    for kind in (0, 1):
        for seed in (1, 55, 1001):
            assert O.gen_scalars(curve, seed, 3000, kind) == kb.gen_scalars(curve, seed, 3000, kind)
    sc = O.gen_scalars(curve, 5, 200)
    edge = [0, 1, 2, 255, 256, 1 << 248, O.FR[curve] - 1, (1 << 254) - 1]
    sc += b"".join(k.to_bytes(32, "little") for k in edge)
    pts = O.fixed_base_points(curve, sc, threads=3)
    pb = O.PB[curve]
    for i in range(len(sc) // 32):
        k = int.from_bytes(sc[32 * i:32 * i + 32], "little")
        assert pts[pb * i:pb * (i + 1)] == O.g1_mul_gen(curve, k), i
