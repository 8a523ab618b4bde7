"""EIP-2537 G1 MSM on the GPU through bls12_381_g1_msm (the reference's
bls/c-abi/c_bls_pairing.cpp:106-110): byte-equal to the oracle, with the
reference's validity rules (range, curve, G1 membership) and its 1/0
return convention."""
from __future__ import annotations

import ctypes
import random

import pytest

import _eip2537 as E
import _oracle as O

pytestmark = pytest.mark.gpu


def kb():
    import crypto_b200
    return crypto_b200


@pytest.mark.parametrize("n,inf_every", [(1, 0), (2, 0), (17, 5), (300, 0), (1000, 9)])
def test_valid_inputs(cuda_lib, n, inf_every):
    rng = random.Random(n)
    xycs, pts, scs = E.valid_input(rng, n, inf_every)
    assert kb().bls12_381_g1_msm(xycs) == (1, E.expected(pts, scs))


def test_matches_plain_msm_at_4096(cuda_lib):
    """Same sum as gpukit_multi_pippenger on the reduced scalars."""
    import torch
    n = 4096
    k = kb()
    sc = k.gen_scalars(2, 17, n)
    ks = k.gen_scalars(2, 18, n)
    d_ks = torch.frombuffer(bytearray(ks), dtype=torch.uint8).cuda()
    d_pts = torch.empty(n * 96, dtype=torch.uint8, device="cuda")
    assert k.lib().kb200_g1_fixed_base_device(2, d_ks.data_ptr(), n, d_pts.data_ptr(), None) == 0
    torch.cuda.synchronize()
    pts = bytes(d_pts.cpu().numpy().tobytes())
    ents = []
    for i in range(n):
        s = int.from_bytes(sc[32 * i:32 * i + 32], "little")
        ents.append(E.entry(pts[96 * i:96 * i + 96], s + (E.R if i % 3 == 0 else 0)))
    rc, out = k.bls12_381_g1_msm(b"".join(ents))
    want = k.gpukit_multi_pippenger(2, sc, pts, n)
    assert rc == 1 and out == bytes(16) + want[:48] + bytes(16) + want[48:]


def test_empty_and_infinity(cuda_lib):
    assert kb().bls12_381_g1_msm(b"") == (1, bytes(128))
    inf = bytes(128) + (5).to_bytes(32, "big")
    assert kb().bls12_381_g1_msm(inf * 4) == (1, bytes(128))
    p = E.g1_point(3)
    assert kb().bls12_381_g1_msm(E.entry(p, E.R)) == (1, bytes(128))
    assert kb().bls12_381_g1_msm(E.entry(p, 0)) == (1, bytes(128))


def test_rejections(cuda_lib):
    rng = random.Random(5)
    good, pts, scs = E.valid_input(rng, 3)
    p = E.g1_point(7)
    x = int.from_bytes(p[:48], "big")
    y = int.from_bytes(p[48:], "big")
    s = (3).to_bytes(32, "big")
    two = E.pad64(0) + E.pad64(2) + s                              # (0, 2) is on the curve
    bad = [
        E.pad64(x + E.P) + E.pad64(y) + s,
        E.pad64(x) + E.pad64(E.P) + s,
        ((1 << 384) | x).to_bytes(64, "big") + E.pad64(y) + s,
        E.pad64(x) + E.pad64((y + 1) % E.P) + s,
        E.entry(E.curve_point_not_in_g1(rng), 3),
        E.entry(E.curve_point_not_in_g1(rng), 0),
        E.entry(E.torsion_point(rng), 3),
        E.pad64(0) + E.pad64(1) + s,
    ]
    for b in bad:
        for data in (good + b, b + good):
            assert O.bls12_381_g1_msm(data)[0] == 0
            assert kb().bls12_381_g1_msm(data)[0] == 0
    assert kb().bls12_381_g1_msm(two)[0] == O.bls12_381_g1_msm(two)[0]
    # a valid call after rejected ones is unaffected
    assert kb().bls12_381_g1_msm(good) == (1, E.expected(pts, scs))


def test_argument_errors(cuda_lib):
    L = kb().lib()
    rx = ctypes.create_string_buffer(64)
    ry = ctypes.create_string_buffer(64)
    good, _, _ = E.valid_input(random.Random(1), 1)
    assert L.bls12_381_g1_msm(rx, ry, good, 159) == 0
    assert L.bls12_381_g1_msm(None, ry, good, 160) == 0
    assert L.bls12_381_g1_msm(rx, ry, None, 160) == 0


def test_device_entry_point(cuda_lib):
    import torch
    rng = random.Random(8)
    xycs, pts, scs = E.valid_input(rng, 64, 6)
    d_in = torch.frombuffer(bytearray(xycs), dtype=torch.uint8).cuda()
    d_out = torch.zeros(96, dtype=torch.uint8, device="cuda")
    d_st = torch.ones(1, dtype=torch.int32, device="cuda")
    assert kb().lib().kb200_bls12_381_g1_msm_device(d_in.data_ptr(), len(xycs), d_out.data_ptr(),
                                                    d_st.data_ptr(), None) == 0
    torch.cuda.synchronize()
    w = E.expected(pts, scs)
    assert int(d_st.item()) == 0
    assert bytes(d_out.cpu().numpy().tobytes()) == w[16:64] + w[80:]
