"""Word-prime NTT on the GPU through the reference's C ABI (ntt_forward /
ntt_inverse, ntt/c-abi/c_ntt.cpp:81-179): bit-exact against the reference's
own known-answer vectors, the fixtures its build produced, and the oracle
across the dispatch, unreduced inputs included."""
from __future__ import annotations

import ctypes
import gzip
import hashlib
import json
import random
import sys
from pathlib import Path

import numpy as np
import pytest

import _oracle as O

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
from make_golden import CYC_Q, CYC_ROOT, GOLD_Q, word_ntt_inputs  # noqa: E402

W = json.load(gzip.open(HERE / "golden" / "word_ntt.json.gz", "rt"))


def kb():
    import crypto_b200
    return crypto_b200


def gpu(x, q, root, inverse=False):
    a = np.array(x, dtype=np.uint64)
    rc = kb().word_ntt_rc(a, len(a), q, root, inverse)
    return rc, a


def test_kat_vectors(cuda_lib):
    for v in W["kat"]:
        rc, f = gpu(v["input"], CYC_Q, CYC_ROOT)
        assert rc == 0 and [int(x) for x in f] == v["forward"], v["name"]
        rc, b = gpu(f, CYC_Q, CYC_ROOT, inverse=True)
        assert rc == 0 and [int(x) for x in b] == v["input"], v["name"]
        # the inverse also accepts the inverse root on the Cyclone path
        rc, b2 = gpu(f, CYC_Q, pow(CYC_ROOT, CYC_Q - 2, CYC_Q), inverse=True)
        assert rc == 0 and np.array_equal(b, b2)


def test_small_path_fixtures(cuda_lib):
    for v in W["small"]:
        rc, f = gpu(v["input"], v["q"], v["root"])
        assert rc == 0 and [int(x) for x in f] == v["forward"], v["name"]
        rc, b = gpu(v["input"], v["q"], v["root"], inverse=True)
        assert rc == 0 and [int(x) for x in b] == v["inverse"], v["name"]


def test_six_step_fixtures(cuda_lib):
    for v in W["large"]:
        x = word_ntt_inputs(v["seed"], v["n"], v["q"], v["canonical"])
        rc, f = gpu(x, v["q"], v["root"])
        assert rc == 0 and hashlib.sha256(f.tobytes()).hexdigest() == v["forward_sha256"], v["name"]
        rc, b = gpu(x, v["q"], v["root_inv"], inverse=True)
        assert rc == 0 and hashlib.sha256(b.tobytes()).hexdigest() == v["inverse_sha256"], v["name"]
        if v["canonical"]:
            rc, rt = gpu(f, v["q"], v["root_inv"], inverse=True)
            assert rc == 0 and np.array_equal(rt, x), v["name"]


@pytest.mark.parametrize("logn", list(range(1, 21)))
def test_sweep_against_oracle(cuda_lib, logn):
    """Every size of the dispatch: Cyclone (pinned root and another root),
    Goldilocks, a 61-bit prime with an arbitrary root, an even and a
    composite modulus, on unreduced 64-bit inputs."""
    n = 1 << logn
    rng = np.random.Generator(np.random.PCG64(logn))
    x = rng.bit_generator.random_raw(n).astype(np.uint64)
    big = logn > 16
    cases = [(CYC_Q, pow(3, (CYC_Q - 1) // (2 * n), CYC_Q) if big else CYC_ROOT),
             (GOLD_Q, pow(7, (GOLD_Q - 1) // ((2 if big else 1) * n), GOLD_Q)),
             ((1 << 61) - 1, 37)]
    if logn <= 12:
        cases += [(CYC_Q, pow(3, (CYC_Q - 1) // n, CYC_Q)), (1 << 40, 12345), (1000003 * 3, 11)]
    for q, root in cases:
        for inv in (False, True):
            rc, got = gpu(x, q, root, inv)
            orc_rc, want = O.word_ntt(x, q, root, inv)
            assert rc == orc_rc == 0
            assert np.array_equal(got, want), (logn, q, root, inv)


def test_round_trips_canonical(cuda_lib):
    """forward then inverse restores canonical input: Cyclone at every size,
    Goldilocks on the six-step path.  (The reference's n <= 2^16 generic path
    adds without an overflow check, ntt/cpp/ntt.cpp:33-37, so for moduli
    above 2^63 it does not round-trip; the sweep above and the fixtures pin
    that behaviour.)"""
    r = random.Random(7)
    for logn in (4, 11, 12, 16, 17, 20):
        n = 1 << logn
        for q, g in ((CYC_Q, 3), (GOLD_Q, 7)):
            if q == GOLD_Q and logn <= 16:
                continue
            root = pow(g, (q - 1) // ((2 if logn > 16 else 1) * n), q)
            if q == CYC_Q and logn <= 16:
                root = CYC_ROOT
            x = np.array([r.randrange(q) for _ in range(n)], dtype=np.uint64)
            rc, f = gpu(x, q, root)
            inv_root = root if (q == CYC_Q and logn <= 16) else pow(root, q - 2, q)
            rc2, b = gpu(f, q, inv_root, inverse=True)
            assert rc == rc2 == 0 and np.array_equal(b, x), (logn, q)


def test_argument_errors(cuda_lib):
    L = kb().lib()
    a = np.arange(8, dtype=np.uint64)
    keep = a.copy()
    assert L.ntt_forward(None, 8, CYC_Q, CYC_ROOT) == -1
    assert L.ntt_forward(a.ctypes.data, 6, CYC_Q, CYC_ROOT) == -1
    assert L.ntt_inverse(a.ctypes.data, 0, CYC_Q, CYC_ROOT) == -1
    assert L.ntt_forward(a.ctypes.data, 8, 0, CYC_ROOT) == -1
    assert np.array_equal(a, keep)  # rejected calls leave the data alone
    big = np.zeros(1 << 17, dtype=np.uint64)
    assert L.ntt_forward(big.ctypes.data, 1 << 17, 0, 3) == -1
    assert L.ntt_forward(big.ctypes.data, 1 << 21, GOLD_Q, 7) == -1
    one = np.array([2 ** 63 + 5], dtype=np.uint64)
    assert L.ntt_inverse(one.ctypes.data, 1, CYC_Q, CYC_ROOT) == 0 and int(one[0]) == 2 ** 63 + 5


def test_device_entry_point(cuda_lib):
    import torch
    n = 1 << 14
    x = word_ntt_inputs(9, n, GOLD_Q, True)
    root = pow(7, (GOLD_Q - 1) // n, GOLD_Q)
    d = torch.from_numpy(x.view(np.int64).copy()).cuda()
    s = torch.empty_like(d)
    L = kb().lib()
    assert L.kb200_word_ntt_device(ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(s.data_ptr()), n,
                                   GOLD_Q, root, 0, None) == 0
    torch.cuda.synchronize()
    _, want = O.word_ntt(x, GOLD_Q, root)
    assert np.array_equal(d.cpu().numpy().view(np.uint64), want)
    # the two-pass sizes need scratch
    assert L.kb200_word_ntt_device(ctypes.c_void_p(d.data_ptr()), None, n, GOLD_Q, root, 0, None) == -1
