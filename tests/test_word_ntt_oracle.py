"""Word-prime NTT oracle (oracle/word_ntt.c) against the reference's own
known-answer vectors (ntt/test/vectors/ntt_kat.json, carried in
tests/golden/word_ntt.json.gz) and against fixtures the reference build
produced across its dispatch (ntt/c-abi/c_ntt.cpp:81-179)."""
from __future__ import annotations

import gzip
import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import _oracle as O

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
from make_golden import CYC_Q, CYC_ROOT, GOLD_Q, word_ntt_inputs  # noqa: E402

W = json.load(gzip.open(HERE / "golden" / "word_ntt.json.gz", "rt"))


def test_kat_forward_and_round_trip():
    for v in W["kat"]:
        rc, f = O.word_ntt(v["input"], CYC_Q, CYC_ROOT)
        assert rc == 0 and [int(x) for x in f] == v["forward"], v["name"]
        rc, b = O.word_ntt(f, CYC_Q, CYC_ROOT, inverse=True)
        assert rc == 0 and [int(x) for x in b] == v["input"], v["name"]


def test_small_path_fixtures():
    for v in W["small"]:
        rc, f = O.word_ntt(v["input"], v["q"], v["root"])
        assert rc == 0 and [int(x) for x in f] == v["forward"], v["name"]
        rc, b = O.word_ntt(v["input"], v["q"], v["root"], inverse=True)
        assert rc == 0 and [int(x) for x in b] == v["inverse"], v["name"]


@pytest.mark.parametrize("idx", [0, 1])
def test_six_step_fixtures(idx):
    v = W["large"][idx]  # the 2^17 cases (2^20 runs in the GPU suite)
    x = word_ntt_inputs(v["seed"], v["n"], v["q"], v["canonical"])
    rc, f = O.word_ntt(x, v["q"], v["root"])
    assert rc == 0 and hashlib.sha256(f.tobytes()).hexdigest() == v["forward_sha256"]
    rc, b = O.word_ntt(x, v["q"], v["root_inv"], inverse=True)
    assert rc == 0 and hashlib.sha256(b.tobytes()).hexdigest() == v["inverse_sha256"]


def test_argument_errors():
    a = np.zeros(8, dtype=np.uint64)
    assert O.orc().orc_word_ntt_forward(None, 8, CYC_Q, CYC_ROOT) == -1
    assert O.orc().orc_word_ntt_forward(a.ctypes.data, 6, CYC_Q, CYC_ROOT) == -1
    assert O.orc().orc_word_ntt_forward(a.ctypes.data, 8, 0, CYC_ROOT) == -1
    big = np.zeros(1 << 17, dtype=np.uint64)
    assert O.orc().orc_word_ntt_forward(big.ctypes.data, 1 << 17, 0, 3) == -1
    assert O.orc().orc_word_ntt_inverse(a.ctypes.data, 1 << 21, CYC_Q, CYC_ROOT) == -1
    one = np.array([12345678901234], dtype=np.uint64)
    assert O.word_ntt(one, GOLD_Q, 1)[1][0] == 12345678901234  # n = 1: untouched


@pytest.mark.skipif(not O.ref_ntt_available(), reason="reference NTT build absent")
def test_oracle_matches_reference_build():
    """Random sweep over the dispatch, unreduced inputs included."""
    import random
    rng = random.Random(3)
    for logn in (1, 3, 6, 9, 12, 16, 17):
        n = 1 << logn
        for q, root in ((CYC_Q, CYC_ROOT), (GOLD_Q, pow(7, (GOLD_Q - 1) // n, GOLD_Q)),
                        ((1 << 61) - 1, 7), (3 * 1000003, 11)):
            if logn > 16:
                root = pow(7, (GOLD_Q - 1) // (2 * n), GOLD_Q) if q == GOLD_Q else root
            x = np.array([rng.getrandbits(64) for _ in range(n)], dtype=np.uint64)
            for inv in (False, True):
                rc, got = O.word_ntt(x, q, root, inv)
                want = x.copy()
                assert O.ref_word_ntt(want, n, q, root, inv) == rc
                assert np.array_equal(got, want), (logn, q, inv)
