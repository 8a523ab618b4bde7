"""Generates the committed golden fixtures in tests/golden/ (run from the repo
root where the reference tree is present):

    make -C oracle all ref && python tests/golden/make_golden.py

MSM expectations come from the reference's own CPU MSM
(gpukit_multi_pippenger_cpu, compiled unmodified into oracle/_ref), with
input points made by the reference's own Montgomery ladder on the generator
(ref_g1_mul_gen).  Sizes follow the reference harness
(gpukit/test/multi_pippenger_test.cpp:37) and its scalar masking (:49-55),
plus full 256-bit scalars at sizes where the reference picks a window of 4
or 8 bits (n = 2, 8, 720), which exercise its dropped top-window carry.

The reference has no Fr NTT, so NTT vectors come from the C restatement in
oracle/ and are cross-checked here against an O(n^2) DFT before writing.
KZG vectors: SRS [tau^i]G1 from the reference ladder, commit = restated iNTT
-> reference MSM -> compressed encoding.

Word-prime NTT vectors (word_ntt.json.gz; `--word-ntt` regenerates only
these): the reference's own known-answer vectors (ntt/test/vectors/
ntt_kat.json, re-checked against the reference build), listed small-size
outputs of the reference build (oracle/_ref/libref_ntt.so) across its
dispatch, and SHA-256 digests of its six-step outputs on seeded inputs.
"""
from __future__ import annotations

import gzip
import json
import os
import random
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
import _oracle as O  # noqa: E402

SEED = 0xC0FFEE


def ref_point(curve: int, k: int) -> bytes:
    import ctypes
    out = ctypes.create_string_buffer(O.PB[curve])
    assert O.ref().ref_g1_mul_gen(curve, k.to_bytes(32, "little"), out) == 0
    return out.raw


def msm_cases(rng: random.Random) -> list[dict]:
    cases = []
    for curve in (1, 2):
        for n, mode in [(1, "masked"), (2, "masked"), (8, "masked"), (64, "masked"),
                        (256, "masked"), (2, "full"), (8, "full"), (720, "full"),
                        (16, "edge")]:
            pts, scs = [], []
            for i in range(n):
                k = rng.getrandbits(252)
                if mode == "edge" and i % 4 == 1:
                    pts.append(bytes(O.PB[curve]))            # infinity point
                elif mode == "edge" and i % 4 == 2 and i > 0:
                    pts.append(pts[i - 2] if pts[i - 2] != bytes(O.PB[curve]) else ref_point(curve, k))
                else:
                    pts.append(ref_point(curve, k))
                s = rng.getrandbits(256)
                if mode == "masked":
                    s &= (1 << 252) - 1                       # top byte & 0x0F
                elif mode == "edge":
                    s = [0, 1, O.FR[curve] - 1, s][i % 4]
                scs.append(s.to_bytes(32, "little"))
            P, S = b"".join(pts), b"".join(scs)
            exp = O.ref_msm(curve, S, P, n)
            assert O.msm(curve, S, P, n) == exp, "restated oracle disagrees with reference"
            cases.append({"curve": curve, "n": n, "mode": mode, "scalars": S.hex(),
                          "points": P.hex(), "expected": exp.hex()})
    return cases


def ntt_cases(rng: random.Random) -> list[dict]:
    cases = []
    for curve in (1, 2):
        for logn in (0, 1, 2, 4, 8):
            n = 1 << logn
            x = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
            for inverse in (0, 1):
                for coset in (0, 1):
                    y = O.ntt(curve, x, bool(inverse), bool(coset))
                    assert y == O.dft(curve, x, bool(inverse), bool(coset))
                    cases.append({"curve": curve, "n": n, "inverse": inverse, "coset": coset,
                                  "input": x.hex(), "expected": y.hex()})
    return cases


def kzg_cases(rng: random.Random) -> list[dict]:
    cases = []
    for n in (1, 4, 16, 64):
        tau = rng.randrange(O.FR[2])
        powers = [pow(tau, i, O.FR[2]) for i in range(n)]
        srs = b"".join(ref_point(2, p) for p in powers)
        ev = b"".join(rng.randrange(O.FR[2]).to_bytes(32, "little") for _ in range(n))
        coeffs = O.ntt(2, ev, inverse=True)
        point = O.ref_msm(2, coeffs, srs, n)
        commit = O.compress(point)
        assert commit == O.kzg_commit(ev, srs)
        cases.append({"n": n, "tau": tau.to_bytes(32, "little").hex(), "srs": srs.hex(),
                      "evals": ev.hex(), "commit": commit.hex()})
    return cases


# ---- word-prime NTT (ntt_forward / ntt_inverse) -----------------------------

CYC_Q, CYC_ROOT = 998244353, 629671588
GOLD_Q = 0xFFFFFFFF00000001
# the reference tree: KINET_REFERENCE, else where the oracle's Makefile looks (REF ?=)
REF_ROOT = Path(os.environ.get("KINET_REFERENCE", "/root/reference"))
KAT = REF_ROOT / "ntt/test/vectors/ntt_kat.json"


def word_ntt_inputs(seed: int, n: int, q: int, canonical: bool):
    """Seeded input words (PCG64 raw 64-bit draws, reduced mod q if
    canonical); the tests regenerate them with this same function."""
    import numpy as np
    raw = np.random.Generator(np.random.PCG64(seed)).bit_generator.random_raw(n).astype(np.uint64)
    return raw % np.uint64(q) if canonical else raw


def ref_word_ntt(words, q: int, root: int, inverse: bool):
    import numpy as np
    a = np.array(words, dtype=np.uint64)
    rc = O.ref_word_ntt(a, len(a), q, root, inverse)
    return rc, a


def word_ntt_cases() -> dict:
    import hashlib
    import numpy as np
    # 1. the reference's own known-answer vectors (Cyclone path), checked
    #    against the reference build before they are copied into the fixture
    kat = []
    for v in json.loads(KAT.read_text()):
        rc, fwd = ref_word_ntt(v["input"], CYC_Q, CYC_ROOT, False)
        assert rc == 0 and [int(x) for x in fwd] == v["forward"], v["name"]
        kat.append({"name": v["name"], "n": v["n"], "input": v["input"], "forward": v["forward"]})
    # 2. listed small-path vectors across the dispatch (reference outputs)
    small = []
    specs = [("cyc_noncanonical", CYC_Q, CYC_ROOT, 256, False),
             ("gold_generic", GOLD_Q, pow(7, (GOLD_Q - 1) // 1024, GOLD_Q), 1024, True),
             ("gold_noncanonical", GOLD_Q, pow(7, (GOLD_Q - 1) // 64, GOLD_Q), 64, False),
             ("cyc_other_root", CYC_Q, pow(3, (CYC_Q - 1) // 512, CYC_Q), 512, True),
             ("mersenne61_any_root", (1 << 61) - 1, 37, 128, False),
             ("even_modulus", 1 << 40, 12345, 32, False)]
    for i, (name, q, root, n, canon) in enumerate(specs):
        x = word_ntt_inputs(100 + i, n, q, canon)
        rc, f = ref_word_ntt(x, q, root, False)
        rc2, b = ref_word_ntt(x, q, root, True)
        assert rc == 0 and rc2 == 0
        small.append({"name": name, "n": n, "q": q, "root": root,
                      "input": [int(v) for v in x], "forward": [int(v) for v in f],
                      "inverse": [int(v) for v in b]})
    # 3. six-step path: hashes of the reference outputs on seeded inputs
    large = []
    for i, (name, q, g, logn, canon) in enumerate([("cyc_2^17", CYC_Q, 3, 17, True),
                                                   ("gold_2^17", GOLD_Q, 7, 17, False),
                                                   ("gold_2^20", GOLD_Q, 7, 20, True),
                                                   ("cyc_2^20", CYC_Q, 3, 20, True)]):
        n = 1 << logn
        root = pow(g, (q - 1) // (2 * n), q)
        x = word_ntt_inputs(200 + i, n, q, canon)
        rc, f = ref_word_ntt(x, q, root, False)
        root_inv = pow(root, q - 2, q)
        rc2, b = ref_word_ntt(x, q, root_inv, True)
        rc3, rt = ref_word_ntt(f, q, root_inv, True)
        assert rc == rc2 == rc3 == 0
        if canon:
            assert np.array_equal(rt, x), name
        large.append({"name": name, "n": n, "q": q, "root": root, "root_inv": root_inv,
                      "seed": 200 + i, "canonical": canon,
                      "forward_sha256": hashlib.sha256(f.tobytes()).hexdigest(),
                      "inverse_sha256": hashlib.sha256(b.tobytes()).hexdigest()})
    return {"kat": kat, "small": small, "large": large}


def main() -> None:
    if "--word-ntt" not in sys.argv[1:]:
        rng = random.Random(SEED)
        data = {"msm": msm_cases(rng), "ntt": ntt_cases(rng), "kzg": kzg_cases(rng)}
        with gzip.open(HERE / "golden.json.gz", "wt") as f:
            json.dump(data, f)
        print({k: len(v) for k, v in data.items()})
    w = word_ntt_cases()
    with gzip.open(HERE / "word_ntt.json.gz", "wt") as f:
        json.dump(w, f)
    print({k: len(v) for k, v in w.items()})


if __name__ == "__main__":
    main()
