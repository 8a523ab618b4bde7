"""EIP-4844 blob commitment and opening proof on the GPU through
kzg_blob_to_commit / kzg_commit_to_proof (the reference's
kzg/c-abi/c_kzg_blob.cpp:26-43), against the oracle's independent route
(monomial setup, inverse NTT, synthetic division) for the same test tau.
Parity with the mainnet setup's bytes is unpinned: neither that setup nor
c-kzg-4844 is available."""
from __future__ import annotations

import random

import pytest

import _blob as B
import _oracle as O

pytestmark = pytest.mark.gpu


def kb():
    import crypto_b200
    return crypto_b200


@pytest.fixture(scope="module")
def setup(cuda_lib):
    assert kb().lib().kzg_blob_setup_generate(B.TAU.to_bytes(32, "little")) == 0
    return B.monomial_srs()


def test_commit(setup):
    for seed in (1, 2):
        blob = B.rand_blob(seed)
        rc, c = kb().kzg_blob_to_commit(blob)
        assert rc == 0 and (0, c) == O.kzg_blob_commit(blob, setup)
    assert kb().kzg_blob_to_commit(bytes(32 * B.N)) == (0, b"\xc0" + bytes(47))


def test_proof_outside_and_inside_domain(setup):
    rng = random.Random(3)
    blob = B.rand_blob(3)
    zs = [rng.randrange(B.R), 0, 1, B.domain_point(0), B.domain_point(1234), B.domain_point(4095)]
    for z in zs:
        zb = z.to_bytes(32, "big")
        rc, proof, y = kb().kzg_commit_to_proof(blob, zb)
        assert rc == 0
        assert (0, proof, y) == O.kzg_blob_proof(blob, zb, setup), z


def test_rejections(setup):
    blob = bytearray(B.rand_blob(5))
    good_z = (12345).to_bytes(32, "big")
    assert kb().kzg_commit_to_proof(bytes(blob), B.R.to_bytes(32, "big"))[0] == -1
    blob[32 * 9:32 * 10] = B.R.to_bytes(32, "big")
    assert kb().kzg_blob_to_commit(bytes(blob))[0] == -1
    assert kb().kzg_commit_to_proof(bytes(blob), good_z)[0] == -1
    L = kb().lib()
    out = bytes(48)
    assert L.kzg_blob_to_commit(None, out) == -1
    # a good call afterwards is unaffected
    good = B.rand_blob(6)
    assert kb().kzg_blob_to_commit(good) == O.kzg_blob_commit(good, setup)


def test_setup_loaded_from_compressed_lagrange_points(setup):
    pts = B.lagrange_compressed()
    L = kb().lib()
    assert L.kzg_blob_setup_load_g1_lagrange(pts, B.N) == 0
    blob = B.rand_blob(7)
    assert kb().kzg_blob_to_commit(blob) == O.kzg_blob_commit(blob, setup)
    z = (987654321).to_bytes(32, "big")
    rc, proof, y = kb().kzg_commit_to_proof(blob, z)
    assert (rc, proof, y) == O.kzg_blob_proof(blob, z, setup)
    # a corrupted point is rejected and leaves no usable setup
    bad = bytearray(pts)
    bad[48 * 10 + 47] ^= 1
    assert L.kzg_blob_setup_load_g1_lagrange(bytes(bad), B.N) == -1
    assert kb().kzg_blob_to_commit(blob)[0] == -1
    assert L.kzg_blob_setup_load_g1_lagrange(pts, B.N - 1) == -2
    # restore for the other tests
    assert L.kzg_blob_setup_generate(B.TAU.to_bytes(32, "little")) == 0
