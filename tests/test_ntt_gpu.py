"""GPU Fr NTT parity (ntt_fr_forward / ntt_fr_inverse via the C ABI) against
the oracle, bit-exact, plus round trips and subsampled DFT checks at large
sizes."""
from __future__ import annotations

import ctypes
import gzip
import json
import random
from pathlib import Path

import numpy as np
import pytest

import _oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden.json.gz"


def kb():
    import crypto_b200
    return crypto_b200


def rand_fr(curve: int, n: int, seed: int) -> bytes:
    return kb().gen_scalars(curve, seed, n)


def test_golden_vectors(cuda_lib):
    with gzip.open(GOLDEN, "rt") as f:
        cases = json.load(f)["ntt"]
    for c in cases:
        got = kb().ntt_fr(c["curve"], bytes.fromhex(c["input"]), bool(c["inverse"]), bool(c["coset"]))
        assert got.hex() == c["expected"], (c["curve"], c["n"], c["inverse"], c["coset"])


@pytest.mark.parametrize("curve", [1, 2])
@pytest.mark.parametrize("logn", list(range(0, 19)))
def test_against_oracle(cuda_lib, curve, logn):
    n = 1 << logn
    x = rand_fr(curve, n, seed=logn * 10 + curve)
    for inverse in (False, True):
        for coset in (False, True):
            assert kb().ntt_fr(curve, x, inverse, coset) == O.ntt(curve, x, inverse, coset), \
                (logn, inverse, coset)


@pytest.mark.parametrize("curve", [1, 2])
def test_non_canonical_inputs_are_reduced(cuda_lib, curve):
    r = O.FR[curve]
    rng = random.Random(1)
    n = 64
    vals = [rng.randrange(r, 1 << 256) for _ in range(n)]
    x = b"".join(v.to_bytes(32, "little") for v in vals)
    xr = b"".join((v % r).to_bytes(32, "little") for v in vals)
    assert kb().ntt_fr(curve, x) == O.ntt(curve, xr)


def _eval_at(curve: int, coeffs: list[int], x: int) -> int:
    r = O.FR[curve]
    acc = 0
    for c in reversed(coeffs):
        acc = (acc * x + c) % r
    return acc


@pytest.mark.parametrize("curve,logn", [(2, 20), (1, 20), (2, 22), (1, 22)])
def test_large_round_trip_and_subsample(cuda_lib, curve, logn):
    n = 1 << logn
    r = O.FR[curve]
    x = rand_fr(curve, n, seed=logn)
    y = kb().ntt_fr(curve, x)
    assert kb().ntt_fr(curve, y, inverse=True) == x
    # Subsample: X_k = p(w^k) by direct evaluation on the CPU.
    buf = ctypes.create_string_buffer(32)
    assert O.orc().orc_root_of_unity(curve, n, buf) == 0
    w = int.from_bytes(buf.raw, "little")
    arr = np.frombuffer(x, dtype=np.uint64).reshape(n, 4)
    coeffs = [int(a) | (int(b) << 64) | (int(c) << 128) | (int(d) << 192) for a, b, c, d in arr]
    for k in (0, 1, n // 3, n - 1):
        assert int.from_bytes(y[32 * k:32 * k + 32], "little") == _eval_at(curve, coeffs, pow(w, k, r))
    # coset round trip
    z = kb().ntt_fr(curve, x, coset=True)
    assert kb().ntt_fr(curve, z, inverse=True, coset=True) == x


def test_errors(cuda_lib):
    L = kb().lib()
    buf = ctypes.create_string_buffer(32 * 3)
    assert L.ntt_fr_forward(2, buf, 3, 0) == -2        # not a power of two
    assert L.ntt_fr_forward(2, None, 4, 0) == -1       # null
    assert L.ntt_fr_forward(7, buf, 2, 0) == -1        # bad curve
    assert L.ntt_fr_forward(1, buf, 1 << 29, 0) == -2  # beyond BN254 2-adicity
