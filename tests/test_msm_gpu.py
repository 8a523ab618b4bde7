"""GPU MSM parity: gpukit_multi_pippenger (CUDA body, via the C ABI) against
the reference's CPU MSM and the committed golden vectors, bit-exact."""
from __future__ import annotations

import ctypes
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


def rand_points(curve: int, n: int, seed: int) -> bytes:
    """n distinct points k_i * G from the CUDA fixed-base path, validated on
    a subsample against the oracle's ladder."""
    import torch
    k = kb()
    sc = k.gen_scalars(curve, seed, n)
    d_sc = torch.frombuffer(bytearray(sc), dtype=torch.uint8).cuda()
    d_pts = torch.empty(n * O.PB[curve], dtype=torch.uint8, device="cuda")
    rc = k.lib().kb200_g1_fixed_base_device(curve, d_sc.data_ptr(), n, d_pts.data_ptr(), None)
    assert rc == 0, k.last_error()
    torch.cuda.synchronize()
    pts = bytes(d_pts.cpu().numpy().tobytes())
    pb = O.PB[curve]
    for i in sorted({0, n // 2, n - 1}):
        kk = int.from_bytes(sc[32 * i:32 * i + 32], "little")
        assert pts[pb * i:pb * (i + 1)] == O.g1_mul_gen(curve, kk), i
    return pts


# The drop-in (exact for every curve point) and the G1-promise entry point
# (GLV split on BLS12-381); every input below is in G1 unless a test says
# otherwise, so both must give the reference's bytes.
PATHS = ["plain", "subgroup"]


def msm(path: str, curve: int, scalars: bytes, points: bytes, n: int) -> bytes:
    if path == "subgroup":
        return kb().gpukit_multi_pippenger_subgroup(curve, scalars, points, n)
    return kb().gpukit_multi_pippenger(curve, scalars, points, n)


@pytest.mark.parametrize("path", PATHS)
def test_golden_vectors(cuda_lib, path):
    with gzip.open(GOLDEN, "rt") as f:
        cases = json.load(f)["msm"]
    for c in cases:
        got = msm(path, c["curve"], bytes.fromhex(c["scalars"]), bytes.fromhex(c["points"]), c["n"])
        assert got.hex() == c["expected"], (c["curve"], c["n"], c["mode"])


@pytest.mark.parametrize("curve,n,frac", [(2, 97, 2), (2, 3000, 3), (2, 1 << 17, 16), (1, 3000, 3)])
def test_points_outside_g1_match_reference(cuda_lib, curve, n, frac):
    """The reference reads any affine curve point with no subgroup check
    (gpukit/curve_traits/bls12_381_g1_first_party_traits.h:58-69), so its
    sum is defined for BLS12-381 points outside G1 too.  The drop-in must
    give its bytes for them: G1 points shifted by points of cofactor order,
    random curve points and pure torsion points, one in `frac` of the
    inputs, at a size with a reference window of 4 or 8 (full 256-bit
    scalars), a mid size and one large enough for the pairing levels.  The
    G1-promise entry point's GLV split is wrong there, which shows the
    drop-in does not take it.  (BN254 has cofactor 1: every point is in G1.)"""
    import _eip2537 as E
    rng = random.Random(n)
    pb = O.PB[curve]
    pts = bytearray(rand_points(curve, n, seed=300 + n))
    if curve == 2:
        tors = [E.torsion_point(rng) for _ in range(4)]
        odd = [E.curve_point_not_in_g1(rng) for _ in range(4)]
        for i in range(0, n, frac):
            kind = rng.randrange(3)
            if kind == 0:
                q = O.g1_add(2, bytes(pts[pb * i:pb * (i + 1)]), tors[rng.randrange(4)])
            elif kind == 1:
                q = odd[rng.randrange(4)]
            else:
                q = tors[rng.randrange(4)]
            pts[pb * i:pb * (i + 1)] = q
    pts = bytes(pts)
    full = n < 128
    S = b"".join((rng.getrandbits(256) if full else rng.randrange(O.FR[curve])).to_bytes(32, "little")
                 for _ in range(n))
    # one reference call below 2^12 points: with full 256-bit scalars its
    # dropped top carry depends on the window it picks for n, so slicing the
    # input (ref_msm_parallel) would change the bytes; above, the scalars are
    # canonical and the sliced run is exact
    if not O.ref_available():
        want = O.msm(curve, S, pts, n)
    elif n <= 4096:
        want = O.ref_msm(curve, S, pts, n)
        assert O.msm(curve, S, pts, n) == want
    else:
        want = O.ref_msm(curve, S, pts, n, threads=16)
    assert kb().gpukit_multi_pippenger(curve, S, pts, n) == want
    out = ctypes.create_string_buffer(O.PB[curve])
    assert kb().lib().gpukit_multi_pippenger_cuda(curve, S, pts, n, out) == 0
    assert out.raw == want
    if curve == 2:
        assert kb().gpukit_multi_pippenger_subgroup(curve, S, pts, n) != want


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("curve", [1, 2])
def test_reference_harness_sizes(cuda_lib, curve, path):
    """Sizes of gpukit/test/multi_pippenger_test.cpp:37 with its scalar mask."""
    rng = random.Random(100 + curve)
    pts_all = rand_points(curve, 4096, seed=31 + curve)
    pb = O.PB[curve]
    for n in (1, 2, 8, 64, 256, 1024, 4096):
        pts = pts_all[:pb * n]
        scs = b"".join((rng.getrandbits(256) & ((1 << 252) - 1)).to_bytes(32, "little")
                       for _ in range(n))
        want = O.ref_msm(curve, scs, pts, n, threads=8) if O.ref_available() else O.msm(curve, scs, pts, n)
        assert msm(path, curve, scs, pts, n) == want, n


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("curve", [1, 2])
def test_full_range_scalars_reproduce_reference_carry(cuda_lib, curve, path):
    """Scalars >= 2^255 at sizes whose reference window is 4 or 8 bits."""
    rng = random.Random(9)
    pts_all = rand_points(curve, 1500, seed=77)
    pb = O.PB[curve]
    for n in (2, 8, 9, 700, 1500):
        pts = pts_all[:pb * n]
        scs = b"".join(rng.getrandbits(256).to_bytes(32, "little") for _ in range(n))
        assert msm(path, curve, scs, pts, n) == O.msm(curve, scs, pts, n), n


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("curve", [1, 2])
def test_edge_cases(cuda_lib, curve, path):
    pb = O.PB[curve]
    r = O.FR[curve]
    g = O.g1_mul_gen(curve, 1)
    p = O.g1_mul_gen(curve, 123456789)
    neg_p = O.g1_mul_gen(curve, r - 123456789)
    zero = bytes(pb)
    cases = [
        ([g], [0]),                                   # zero scalar -> identity
        ([zero], [5]),                                # identity point
        ([p, p, p, p], [3, 3, 3, 3]),                 # same point in one bucket (doubling)
        ([p, neg_p], [7, 7]),                         # P + (-P) in one bucket -> infinity
        ([p, neg_p, g], [7, 7, 1]),
        ([g] * 64, [1] * 64),                         # every entry in one bucket
        ([g, p], [r - 1, r]),                         # r - 1 and r itself
        ([g, p], [(1 << 256) - 1, 1 << 255]),         # top of the 256-bit range
    ]
    for pts, scs in cases:
        P = b"".join(pts)
        S = b"".join(s.to_bytes(32, "little") for s in scs)
        assert msm(path, curve, S, P, len(pts)) == O.msm(curve, S, P, len(pts))


def test_n_zero_and_errors(cuda_lib):
    k = kb()
    out = ctypes.create_string_buffer(96)
    assert k.msm_rc(2, None, None, 0, out) == 0
    assert out.raw == bytes(96)
    assert k.msm_rc(2, None, None, 1, out) == -1          # GPUKIT_ERR_NULL_ARG
    assert k.msm_rc(2, b"\0" * 32, b"\0" * 96, 1, None) == -1
    assert k.msm_rc(0, b"\0" * 32, b"\0" * 64, 1, out) == -5   # secp256k1: NOTIMPL
    assert k.msm_rc(3, b"\0" * 32, b"\0" * 64, 1, out) == -5   # banderwagon: NOTIMPL
    assert k.msm_rc(9, b"\0" * 32, b"\0" * 64, 1, out) == -3   # unknown: BACKEND
    L = k.lib()
    assert L.gpukit_multi_pippenger_subgroup(2, None, None, 0, out) == 0
    assert out.raw == bytes(96)
    assert L.gpukit_multi_pippenger_subgroup(2, None, None, 1, out) == -1
    assert L.gpukit_multi_pippenger_subgroup(0, b"\0" * 32, b"\0" * 64, 1, out) == -5
    assert L.gpukit_multi_pippenger_subgroup(9, b"\0" * 32, b"\0" * 64, 1, out) == -3


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("curve", [1, 2])
def test_skewed_scalars(cuda_lib, curve, path):
    """50% of scalars in {0,1}, 20% below 2^64, rest uniform (bucket imbalance)."""
    n = 1 << 14
    pts = rand_points(curve, n, seed=5)
    scs = kb().gen_scalars(curve, 1234, n, kind=1)
    want = O.ref_msm(curve, scs, pts, n, threads=8) if O.ref_available() else O.msm(curve, scs, pts, n)
    assert msm(path, curve, scs, pts, n) == want


@pytest.mark.parametrize("path", PATHS)
def test_skewed_scalars_tiled_ranking(cuda_lib, path):
    """Skewed scalars at a size whose sort ranks by tiles (BLS12-381, 2^17
    points: over 2^20 entries, windows of at most 2^15 buckets): the hot
    buckets of the {0, 1} scalars meet in a tile's shared counters through
    the warp's grouping of equal keys; the bytes equal the reference's."""
    n = 1 << 17
    pts = rand_points(2, n, seed=6)
    scs = kb().gen_scalars(2, 4321, n, kind=1)
    want = O.ref_msm(2, scs, pts, n, threads=16) if O.ref_available() else O.msm(2, scs, pts, n)
    assert msm(path, 2, scs, pts, n) == want


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("curve", [1, 2])
def test_2_16_against_reference(cuda_lib, curve, path):
    n = 1 << 16
    pts = rand_points(curve, n, seed=8)
    scs = kb().gen_scalars(curve, 4321, n)
    want = O.ref_msm(curve, scs, pts, n, threads=8) if O.ref_available() else O.msm(curve, scs, pts, n)
    assert msm(path, curve, scs, pts, n) == want


@pytest.mark.parametrize("curve", [1, 2])
def test_linearity_large(cuda_lib, curve):
    """Size-independent property at a large size: MSM(s, P) + MSM(t, P) ==
    MSM(s + t mod r, P), and splitting the input gives the same sum."""
    n = 1 << 18
    pts = rand_points(curve, n, seed=21)
    s = kb().gen_scalars(curve, 1, n)
    t = kb().gen_scalars(curve, 2, n)
    r = O.FR[curve]
    st = b"".join(((int.from_bytes(s[32 * i:32 * i + 32], "little") +
                    int.from_bytes(t[32 * i:32 * i + 32], "little")) % r).to_bytes(32, "little")
                  for i in range(n))
    a = kb().gpukit_multi_pippenger(curve, s, pts, n)
    b = kb().gpukit_multi_pippenger(curve, t, pts, n)
    c = kb().gpukit_multi_pippenger(curve, st, pts, n)
    assert O.g1_add(curve, a, b) == c
    pb = O.PB[curve]
    h = n // 2
    lo = kb().gpukit_multi_pippenger(curve, s[:32 * h], pts[:pb * h], h)
    hi = kb().gpukit_multi_pippenger(curve, s[32 * h:], pts[pb * h:], n - h)
    assert O.g1_add(curve, lo, hi) == a


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("curve,logn,bits", [(1, 20, 10), (2, 18, 8)])
def test_many_big_buckets(cuda_lib, curve, logn, bits, path):
    """Small scalars over many points: every bucket of window 0 holds
    thousands of entries, so thousands of buckets take the fold path."""
    n = 1 << logn
    pts = rand_points(curve, n, seed=40 + logn)
    rng = random.Random(logn)
    scs = b"".join(rng.getrandbits(bits).to_bytes(32, "little") for _ in range(n))
    want = O.ref_msm(curve, scs, pts, n, threads=16) if O.ref_available() else O.msm(curve, scs, pts, n)
    assert msm(path, curve, scs, pts, n) == want


def test_glv_halves_share_a_bucket(cuda_lib):
    """Scalars a + a*lambda: both GLV halves carry the same small digit, so
    one bucket of window 0 receives 2n entries (the planner's largest-bucket
    bound must count both halves)."""
    lam = 0xAC45A4010001A40200000000FFFFFFFF
    n = 1 << 14
    pts = rand_points(2, n, seed=66)
    rng = random.Random(66)
    scs = []
    for i in range(n):
        a = 3 if i % 10 else rng.randrange(1, 200)  # bucket 3 gets ~1.8 n entries
        scs.append(((a + a * lam) % O.FR[2]).to_bytes(32, "little"))
    S = b"".join(scs)
    want = O.ref_msm(2, S, pts, n, threads=16) if O.ref_available() else O.msm(2, S, pts, n)
    assert kb().gpukit_multi_pippenger_subgroup(2, S, pts, n) == want
    assert kb().gpukit_multi_pippenger(2, S, pts, n) == want


def test_bn254_glv_halves_signs_and_bounds(cuda_lib):
    """BN254 splits every scalar as k = k1 + k2 lambda with signed halves
    (Babai rounding).  Scalars near the rounding boundaries of the split --
    k = round(j r / b) for the basis entries b, their neighbours, multiples
    of lambda and the range ends -- give the reference's bytes."""
    r = O.FR[1]
    lam = 0xB3C4D79D41A917585BFC41088D8DAAA78B17EA66B99C90DD
    b1 = 0x6F4D8248EEB859FC8211BBEB7D4F1128
    b2 = 0x89D3256894D213E3
    ks = {0, 1, 2, r - 1, r - 2, lam, lam - 1, lam + 1, (r - 1) // 2, (r + 1) // 2}
    rng = random.Random(254)
    for b in (b1, b2):
        for _ in range(300):
            j = rng.randrange(1, b)
            c = (2 * j + 1) * r // (2 * b)  # k b / r just below / above j + 1/2
            ks.update({c % r, (c + 1) % r, (c - 1) % r})
    for _ in range(100):
        ks.add(rng.randrange(1, 1 << 64) * lam % r)
    ks = sorted(ks)
    n = len(ks)
    pts = rand_points(1, n, seed=254)
    S = b"".join(k.to_bytes(32, "little") for k in ks)
    want = O.ref_msm(1, S, pts, n, threads=8) if O.ref_available() else O.msm(1, S, pts, n)
    assert kb().gpukit_multi_pippenger(1, S, pts, n) == want
    # a sample of the scalars alone (n = 1: a single point per MSM)
    for i in range(0, n, 97):
        assert kb().gpukit_multi_pippenger(1, S[32 * i:32 * i + 32], pts[64 * i:64 * i + 64], 1) == \
            O.msm(1, S[32 * i:32 * i + 32], pts[64 * i:64 * i + 64], 1)


@pytest.mark.parametrize("levels", [1, 4])
def test_pairing_levels_bit_exact(cuda_lib, levels):
    """The batch-affine pairing levels, forced (KB200_MSM_PAIR_LEVELS) on
    inputs whose runs the planner would not pair, give the same bytes: long
    runs in a few buckets, repeated points (doublings) and cancelling pairs
    (infinity rows that later levels pass through)."""
    import os
    import subprocess
    import sys
    code = r'''
import random, sys
sys.path.insert(0, "tests")
import crypto_b200 as kb, _oracle as O
for curve, n in ((2, 1 << 13), (1, 1 << 13)):
    rng = random.Random(curve)
    base = [O.g1_mul_gen(curve, rng.randrange(1, O.FR[curve])) for _ in range(64)]
    pts, scs = [], []
    for i in range(n):
        p = base[i % 64]
        if i % 5 == 1:
            p = pts[-1]                                # repeated point in the same bucket
        if i % 11 == 2:
            p = O.g1_mul(curve, pts[-1], O.FR[curve] - 1)  # its negation: cancels
        pts.append(p)
        scs.append(rng.choice((1, 2, 3, 7, 1 << 70)).to_bytes(32, "little"))
    P, S = b"".join(pts), b"".join(scs)
    want = O.msm(curve, S, P, n)
    assert kb.gpukit_multi_pippenger(curve, S, P, n) == want, curve
    assert kb.gpukit_multi_pippenger_subgroup(curve, S, P, n) == want, curve
print("ok")
'''
    env = dict(os.environ, KB200_MSM_PAIR_LEVELS=str(levels))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0 and "ok" in out.stdout, out.stdout + out.stderr


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("curve,logn", [(2, 20), (1, 17), (1, 20)])
def test_host_pipeline_with_infinity_points(cuda_lib, curve, logn, path):
    """gpukit_multi_pippenger copies the scalars and the points in row chunks
    (four at these sizes), sorting and pairing each chunk as it lands when the
    plan pairs, and converts each point chunk on its own stream, so infinity
    points reach the buckets and are skipped there: one point in eight is
    the identity (and, at 2^20 on BLS12-381, with pairing levels)."""
    n = 1 << logn
    pb = O.PB[curve]
    pts = bytearray(rand_points(curve, n, seed=90 + curve))
    rng = random.Random(90 + curve)
    for i in range(0, n, 8):
        j = i + rng.randrange(8)
        pts[pb * j:pb * (j + 1)] = bytes(pb)
    pts = bytes(pts)
    S = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
    want = O.ref_msm(curve, S, pts, n, threads=16) if O.ref_available() else O.msm(curve, S, pts, n)
    assert msm(path, curve, S, pts, n) == want


@pytest.mark.parametrize("curve", [1, 2])
def test_device_entry_aligned_and_unaligned_points(cuda_lib, curve):
    """kb200_msm_device reads wire points straight from device memory: in
    16-byte pieces from an aligned base, byte by byte from any other (here
    one byte past an aligned allocation); both give the oracle's bytes, with
    infinity points among the inputs."""
    import torch
    n = 3001
    pb = O.PB[curve]
    pts = bytearray(rand_points(curve, n, seed=120 + curve))
    for j in (0, 17, n - 1):
        pts[pb * j:pb * (j + 1)] = bytes(pb)
    pts = bytes(pts)
    rng = random.Random(120 + curve)
    S = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
    want = O.msm(curve, S, pts, n)
    d_sc = torch.frombuffer(bytearray(S), dtype=torch.uint8).cuda()
    d_out = torch.empty(pb, dtype=torch.uint8, device="cuda")
    for shift in (0, 1):
        buf = torch.zeros(n * pb + 16, dtype=torch.uint8, device="cuda")
        buf[shift:shift + n * pb] = torch.frombuffer(bytearray(pts), dtype=torch.uint8).cuda()
        for fn in (kb().lib().kb200_msm_device, kb().lib().kb200_msm_device_subgroup):
            d_out.zero_()
            rc = fn(curve, d_sc.data_ptr(), buf.data_ptr() + shift, n, d_out.data_ptr(), None)
            assert rc == 0, kb().last_error()
            torch.cuda.synchronize()
            assert bytes(d_out.cpu().numpy().tobytes()) == want, shift


@pytest.mark.parametrize("quad,curve,logn", [(1, 2, 20), (1, 1, 17), (0, 2, 12), (0, 1, 14)])
def test_reduction_modes_bit_exact(cuda_lib, quad, curve, logn):
    """The bucket reduction has a quad-lane form for few buckets and the
    per-thread form for many; forcing each where the planner picks the other
    (KB200_MSM_RED_QUAD) gives the oracle's bytes: the quad form with several
    buckets per slot over many windows, the per-thread form at small sizes."""
    import os
    import subprocess
    import sys
    code = r'''
import random, sys
sys.path.insert(0, "tests")
import crypto_b200 as kb, _oracle as O
from test_msm_gpu import rand_points
curve, logn = %d, %d
n = 1 << logn
pts = rand_points(curve, n, seed=140 + logn)
rng = random.Random(140 + logn)
S = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
want = O.ref_msm(curve, S, pts, n, threads=16) if O.ref_available() else O.msm(curve, S, pts, n)
assert kb.gpukit_multi_pippenger(curve, S, pts, n) == want
print("ok")
''' % (curve, logn)
    env = dict(os.environ, KB200_MSM_RED_QUAD=str(quad))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0 and "ok" in out.stdout, out.stdout + out.stderr


@pytest.mark.parametrize("chunks", [3, 8])
@pytest.mark.parametrize("curve", [1, 2])
def test_host_pipeline_uneven_chunks(cuda_lib, curve, chunks):
    """Row chunks that do not divide n (3: the last chunk shorter) and the
    largest count (8): each scalar chunk's recode and ranking cover exactly
    its rows (KB200_MSM_HOST_CHUNKS), with infinity points among the inputs;
    the bytes equal the reference's."""
    import os
    import subprocess
    import sys
    code = r'''
import random, sys
sys.path.insert(0, "tests")
import crypto_b200 as kb, _oracle as O
from test_msm_gpu import rand_points
curve = %d
n = (1 << 17) + 5
pb = O.PB[curve]
pts = bytearray(rand_points(curve, n, seed=160 + curve))
for j in (0, 1, n // 3, n - 1):
    pts[pb * j:pb * (j + 1)] = bytes(pb)
pts = bytes(pts)
rng = random.Random(160 + curve)
S = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
want = O.ref_msm(curve, S, pts, n, threads=16) if O.ref_available() else O.msm(curve, S, pts, n)
for path in ("plain", "subgroup"):
    f = kb.gpukit_multi_pippenger if path == "plain" else kb.gpukit_multi_pippenger_subgroup
    assert f(curve, S, pts, n) == want, path
print("ok")
''' % curve
    env = dict(os.environ, KB200_MSM_HOST_CHUNKS=str(chunks))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0 and "ok" in out.stdout, out.stdout + out.stderr


@pytest.mark.parametrize("chunks", [3, 7])
@pytest.mark.parametrize("curve", [1, 2])
def test_host_pipeline_pairs_per_uneven_chunk(cuda_lib, curve, chunks):
    """At a size whose plan pairs (2^20 + 3 points) the host pipeline sorts
    and pairs each row chunk once its own scalars and points are resident:
    chunk scans chained on the device, first-level sums at their entry
    positions, level 1 through the chunks' index.  Row chunks that do not
    divide n, infinity points and repeated points among the inputs; the
    bytes equal the reference's."""
    import os
    import subprocess
    import sys
    code = r'''
import random, sys
sys.path.insert(0, "tests")
import crypto_b200 as kb, _oracle as O
from test_msm_gpu import rand_points
curve = %d
n = (1 << 20) + 3
pb = O.PB[curve]
pts = bytearray(rand_points(curve, n, seed=170 + curve))
rng = random.Random(170 + curve)
for j in rng.sample(range(n), 64):
    pts[pb * j:pb * (j + 1)] = bytes(pb)
for j in rng.sample(range(1, n), 64):
    pts[pb * j:pb * (j + 1)] = pts[pb * (j - 1):pb * j]
pts = bytes(pts)
S = b"".join(rng.randrange(O.FR[curve]).to_bytes(32, "little") for _ in range(n))
want = O.ref_msm(curve, S, pts, n, threads=16) if O.ref_available() else O.msm(curve, S, pts, n)
for path in ("plain", "subgroup"):
    f = kb.gpukit_multi_pippenger if path == "plain" else kb.gpukit_multi_pippenger_subgroup
    assert f(curve, S, pts, n) == want, path
print("ok")
''' % curve
    env = dict(os.environ, KB200_MSM_HOST_CHUNKS=str(chunks))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                         text=True, timeout=1200)
    assert out.returncode == 0 and "ok" in out.stdout, out.stdout + out.stderr
