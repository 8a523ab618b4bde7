"""GPU KZG commit parity: synthetic SRS generation and kzg_commit_fr /
kzg_commit_batch against the oracle (restated iNTT -> reference MSM ->
compressed encoding), byte-exact."""
from __future__ import annotations

import gzip
import json
import random
from pathlib import Path

import pytest

import _oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden.json.gz"


def kb():
    import crypto_b200
    return crypto_b200


def test_golden_commits(cuda_lib):
    with gzip.open(GOLDEN, "rt") as f:
        cases = json.load(f)["kzg"]
    for c in cases:
        kb().kzg_srs_load(bytes.fromhex(c["srs"]))
        assert kb().kzg_commit(bytes.fromhex(c["evals"])).hex() == c["commit"], c["n"]
        # the generated SRS from the same tau equals the loaded one
        kb().kzg_srs_generate(bytes.fromhex(c["tau"]), c["n"])
        assert kb().kzg_srs_read(0, c["n"]) == bytes.fromhex(c["srs"])


def test_srs_generation_subsample(cuda_lib):
    rng = random.Random(4)
    tau = rng.randrange(O.FR[2])
    n = 1 << 16
    kb().kzg_srs_generate(tau.to_bytes(32, "little"), n)
    assert kb().kzg_srs_size() == n
    for i in (0, 1, 2, 4095, n - 1):
        pt = kb().kzg_srs_read(i, 1)
        assert pt == O.g1_mul_gen(2, pow(tau, i, O.FR[2])), i


@pytest.mark.parametrize("n", [1, 2, 256, 4096])
def test_commit_matches_oracle(cuda_lib, n):
    rng = random.Random(n)
    tau = rng.randrange(O.FR[2])
    kb().kzg_srs_generate(tau.to_bytes(32, "little"), max(n, 1))
    srs = kb().kzg_srs_read(0, n)
    ev = kb().gen_scalars(2, 99 + n, n)
    want = O.kzg_commit(ev, srs)
    assert kb().kzg_commit(ev) == want
    if O.ref_available():
        coeffs = O.ntt(2, ev, inverse=True)
        assert O.compress(O.ref_msm(2, coeffs, srs, n, threads=8)) == want


def test_batch_equals_single(cuda_lib):
    rng = random.Random(12)
    tau = rng.randrange(O.FR[2])
    kb().kzg_srs_generate(tau.to_bytes(32, "little"), 1 << 12)
    sizes = [1 << rng.randint(0, 12) for _ in range(24)]
    evs = [kb().gen_scalars(2, 500 + i, s) for i, s in enumerate(sizes)]
    batch = kb().kzg_commit_batch(b"".join(evs), sizes)
    for e, c in zip(evs, batch):
        assert kb().kzg_commit(e) == c


def test_batch_graph_after_engine_growth(cuda_lib):
    """A batch shape is captured into a CUDA graph on first use; a later,
    larger shape grows the shared engine and batch buffers, so replaying the
    first shape must not reuse addresses from before the growth."""
    rng = random.Random(21)
    tau = rng.randrange(O.FR[2])
    kb().kzg_srs_generate(tau.to_bytes(32, "little"), 1 << 16)
    small = [256, 1024, 256]
    large = [1 << 16] * 4 + [1 << 12]
    ev_s = [kb().gen_scalars(2, 900 + i, s) for i, s in enumerate(small)]
    ev_l = [kb().gen_scalars(2, 950 + i, s) for i, s in enumerate(large)]
    want_s = [kb().kzg_commit(e) for e in ev_s]
    want_l = [kb().kzg_commit(e) for e in ev_l]
    for shape, evs, want in [(small, ev_s, want_s), (large, ev_l, want_l), (small, ev_s, want_s),
                             (large, ev_l, want_l), (small, ev_s, want_s)]:
        assert kb().kzg_commit_batch(b"".join(evs), shape) == want


def test_commit_errors(cuda_lib):
    import ctypes
    L = kb().lib()
    kb().kzg_srs_generate((5).to_bytes(32, "little"), 16)
    out = ctypes.create_string_buffer(48)
    assert L.kzg_commit_fr(b"\0" * 32 * 32, 32, out) == -2   # longer than the SRS
    assert L.kzg_commit_fr(b"\0" * 32 * 3, 3, out) == -2     # not a power of two
    assert L.kzg_commit_fr(None, 4, out) == -1
    # zero polynomial commits to infinity (0xC0 || 0...)
    assert kb().kzg_commit(b"\0" * 32 * 16) == b"\xc0" + bytes(47)


def test_commit_with_every_window_in_one_bucket(cuda_lib):
    """Coefficients whose digit is 1 in every window of the shifted-table
    MSM: all W n entries land in one shared bucket (the planner's
    largest-bucket bound must count every window)."""
    n = 4096
    rng = random.Random(77)
    tau = rng.randrange(O.FR[2])
    kb().kzg_srs_generate(tau.to_bytes(32, "little"), n)
    srs = kb().kzg_srs_read(0, n)
    coeffs = []
    for i in range(n):
        c = [13, 16, 19][i % 3]  # every window size the shifted tables use
        v = sum(1 << (c * w) for w in range(255 // c))
        coeffs.append((v % O.FR[2]).to_bytes(32, "little"))
    ev = O.ntt(2, b"".join(coeffs))          # evaluations of that polynomial
    want = O.compress(O.msm(2, b"".join(coeffs), srs, n))
    assert kb().kzg_commit(ev) == want
