"""EIP-2537 G1 MSM oracle (orc_bls12_381_g1_msm) against its definition:
the reference (bls/cpp/bls.cpp:194-254) hands the arithmetic to blst, which
is absent, so the oracle is pinned against the reference's own G1 MSM
(gpukit_multi_pippenger_cpu, through the repacking of
gpukit/curve_traits/bls12_381_g1_traits.h:37-65) and against independent
Python big-integer checks of each rejection rule."""
from __future__ import annotations

import random

import _eip2537 as E
import _oracle as O


def test_valid_inputs_match_reference_msm():
    rng = random.Random(11)
    for n, inf_every in ((1, 0), (3, 0), (16, 4), (40, 7)):
        xycs, pts, scs = E.valid_input(rng, n, inf_every)
        rc, out = O.bls12_381_g1_msm(xycs)
        assert rc == 1
        if O.ref_available() and pts:
            ref = O.ref_msm(2, b"".join(s.to_bytes(32, "little") for s in scs), b"".join(pts), len(pts))
            assert out == bytes(16) + ref[:48] + bytes(16) + ref[48:]
        assert out == E.expected(pts, scs)


def test_empty_and_all_infinity():
    assert O.bls12_381_g1_msm(b"") == (1, bytes(128))
    inf = bytes(128) + (5).to_bytes(32, "big")
    assert O.bls12_381_g1_msm(inf * 3) == (1, bytes(128))


def test_rejections():
    rng = random.Random(12)
    good, _, _ = E.valid_input(rng, 2)
    p = E.g1_point(7)
    x = int.from_bytes(p[:48], "big")
    y = int.from_bytes(p[48:], "big")
    s = (3).to_bytes(32, "big")
    bad = [
        E.pad64(x + E.P) + E.pad64(y) + s,                      # x >= p
        E.pad64(x) + E.pad64(E.P) + s,                          # y = p
        (1 << 400 | x).to_bytes(64, "big") + E.pad64(y) + s,    # top bytes non-zero
        E.pad64(x) + E.pad64((y + 1) % E.P) + s,                # off the curve
        E.entry(E.curve_point_not_in_g1(rng), 3),               # on E, not in G1
        E.entry(E.torsion_point(rng), 3),                       # cofactor torsion
        E.pad64(0) + E.pad64(1) + s,                            # (0,1): not infinity
    ]
    for b in bad:
        assert O.bls12_381_g1_msm(good + b)[0] == 0
        assert O.bls12_381_g1_msm(b + good)[0] == 0
    assert O.bls12_381_g1_msm(good[:159])[0] == 0            # size not a multiple of 160


def test_scalars_reduced_mod_r():
    p = E.g1_point(99)
    a = O.bls12_381_g1_msm(E.entry(p, 5))
    b = O.bls12_381_g1_msm(E.entry(p, 5 + E.R))
    c = O.bls12_381_g1_msm(E.entry(p, 5 + 2 * E.R))
    assert a == b == c and a[0] == 1
    z = O.bls12_381_g1_msm(E.entry(p, E.R))
    assert z == (1, bytes(128))
