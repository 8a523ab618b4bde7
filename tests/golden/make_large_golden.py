"""Generates tests/golden/large.json: expected outputs at the full workload
sizes (run from the repo root where the reference tree is present):

    make -C oracle all ref && python tests/golden/make_large_golden.py

Each MSM case is a seeded workload -- scalars from the library's xorshift64*
streams (restated in the oracle as orc_gen_scalars), points s_i * G with
seeded s_i (orc_g1_fixed_base_batch) -- whose expected sum comes from the
reference's own CPU MSM (gpukit_multi_pippenger_cpu, compiled unmodified into
oracle/_ref) run on contiguous slices in parallel and summed with the
reference g1_add (ref_msm_parallel; byte-identical to one call by the group
law, since every scalar is below r).  The case records SHA-256 digests of the
scalar and point bytes, so a test that rebuilds the inputs another way (the
device fixed-base kernel) proves it rebuilt the same workload.

Each Fr NTT case records SHA-256 digests of the oracle's full forward and
inverse outputs (oracle/oracle.c orc_ntt, the radix-2 restatement) on a
seeded input.  The reference has no Fr NTT, so these are pinned to the
restatement, which is itself checked against an O(n^2) DFT in
tests/test_oracle.py.

Seeds and sizes are the benchmark's (bench.py): the 2^22 BLS12-381 MSM
headline, the 2^20 BLS12-381 MSM, the BN254 2^24 MSMs (uniform and skewed
scalars), the BLS12-381 2^24 NTT and the BN254 2^26 coset NTT.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
import _oracle as O  # noqa: E402

# (label, curve, log2 n, scalar seed, scalar kind, point-scalar seed)
MSM_CASES = [
    ("msm_bls12_381_2^22", 2, 22, 1, 0, 1001),
    ("msm_bls12_381_2^20", 2, 20, 51, 0, 97),
    ("msm_bn254_2^24_uniform", 1, 24, 55, 0, 101),
    ("msm_bn254_2^24_skewed", 1, 24, 55, 1, 101),
]
# (label, curve, log2 n, input seed, coset)
NTT_CASES = [
    ("ntt_bls12_381_2^24", 2, 24, 29, 0),
    ("ntt_bn254_2^26_coset", 1, 26, 31, 1),
]


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def msm_workload(curve: int, logn: int, seed: int, kind: int, pseed: int):
    n = 1 << logn
    scs = O.gen_scalars(curve, seed, n, kind)
    pts = O.fixed_base_points(curve, O.gen_scalars(curve, pseed, n))
    return scs, pts


def main() -> None:
    threads = os.cpu_count() or 1
    out = {"msm": [], "ntt": [], "threads": threads}
    only = set(sys.argv[1:])
    for label, curve, logn, seed, kind, pseed in MSM_CASES:
        if only and label not in only:
            continue
        t0 = time.time()
        scs, pts = msm_workload(curve, logn, seed, kind, pseed)
        t1 = time.time()
        want = O.ref_msm(curve, scs, pts, 1 << logn, threads=threads)
        t2 = time.time()
        out["msm"].append({"label": label, "curve": curve, "log_n": logn, "scalar_seed": seed,
                           "kind": kind, "point_seed": pseed, "scalars_sha256": sha(scs),
                           "points_sha256": sha(pts), "expected": want.hex()})
        print(f"{label}: inputs {t1 - t0:.1f} s, reference MSM ({threads} slices) {t2 - t1:.1f} s",
              flush=True)
    for label, curve, logn, seed, coset in NTT_CASES:
        if only and label not in only:
            continue
        t0 = time.time()
        x = O.gen_scalars(curve, seed, 1 << logn)
        fwd = O.ntt(curve, x, inverse=False, coset=bool(coset))
        inv = O.ntt(curve, x, inverse=True, coset=bool(coset))
        assert O.ntt(curve, fwd, inverse=True, coset=bool(coset)) == x
        out["ntt"].append({"label": label, "curve": curve, "log_n": logn, "seed": seed,
                           "coset": coset, "input_sha256": sha(x), "forward_sha256": sha(fwd),
                           "inverse_sha256": sha(inv), "forward_head": fwd[:64].hex(),
                           "inverse_head": inv[:64].hex()})
        print(f"{label}: oracle forward + inverse + round trip {time.time() - t0:.1f} s", flush=True)
    path = HERE / "large.json"
    if only and path.exists():
        old = json.loads(path.read_text())
        for k in ("msm", "ntt"):
            keep = [c for c in old[k] if c["label"] not in {d["label"] for d in out[k]}]
            out[k] = keep + out[k]
    path.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
