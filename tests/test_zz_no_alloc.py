"""The allocation-free Fr NTT (ntt_fr_transform_noalloc) against the regular
entry points, through the C ABI.

Callers that cannot allocate device memory -- code running during CUDA
graph capture, latency-critical paths that cannot afford cudaMalloc's
implicit synchronisation, processes whose device memory belongs to another
allocator -- use this variant; its scratch lives in a fixed static device
array (n <= 2^16).  Results must be bit-identical to ntt_fr_forward /
ntt_fr_inverse, on consecutive calls that reuse the shared array.  This file
is collected last so a failure here leaves every other test already run.
"""
from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu


def kb():
    import crypto_b200
    return crypto_b200


@pytest.mark.parametrize("curve", [1, 2])
def test_noalloc_matches_regular_two_calls(cuda_lib, curve):
    cases = [(1 << 16, False, False, 11), (1 << 10, True, True, 12),
             (1 << 13, True, False, 13), (1 << 16, False, True, 14)]
    # two calls in a row, then the rest: each reuses the same static array
    for n, inverse, coset, seed in cases:
        x = kb().gen_scalars(curve, seed + curve, n)
        want = kb().ntt_fr(curve, x, inverse=inverse, coset=coset)
        assert kb().ntt_fr_noalloc(curve, x, inverse=inverse, coset=coset) == want, (n, inverse, coset)


def test_noalloc_rejects_beyond_limit(cuda_lib):
    n = 1 << 17
    buf = ctypes.create_string_buffer(32)  # never read: the size check comes first
    assert kb().lib().ntt_fr_transform_noalloc(2, buf, n, 0, 0) == -2
    assert "2^16" in kb().last_error()
    assert kb().lib().ntt_fr_transform_noalloc(2, buf, 3, 0, 0) == -2
