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
"""
from __future__ import annotations

import gzip
import json
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


def main() -> None:
    rng = random.Random(SEED)
    data = {"msm": msm_cases(rng), "ntt": ntt_cases(rng), "kzg": kzg_cases(rng)}
    with gzip.open(HERE / "golden.json.gz", "wt") as f:
        json.dump(data, f)
    print({k: len(v) for k, v in data.items()})


if __name__ == "__main__":
    main()
