"""The allocation-free Fr NTT (ntt_fr_transform_noalloc) against the regular
entry points, through the C ABI.

ntt_fr_forward / ntt_fr_inverse grow device scratch with cudaMalloc when
they meet a new size.  Callers whose device memory is reserved up front by
another allocator (a framework's caching pool, a fixed arena), or that cannot
afford the device-wide waits of cudaMalloc and cudaFree, use this variant
instead: its scratch lives in a fixed static device array (n <= 2^16).  Its
results must be bit-identical to the regular entry points', on consecutive
calls that reuse the shared array, and a call on a warm device must leave
the device's free memory unchanged.  This file is collected last so a
failure here leaves every other test already run.
"""
from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu


def kb():
    import crypto_b200
    return crypto_b200


# (n, inverse, coset, seed): single-pass sizes from one element up, the
# two-pass sizes, the largest allowed
CASES = [(1 << 16, False, False, 11), (1 << 10, True, True, 12), (1 << 13, True, False, 13),
         (1 << 16, False, True, 14), (1, False, False, 15), (1, True, True, 16), (2, False, True, 17),
         (2, True, False, 18), (4, True, True, 19), (4, False, False, 20)]


@pytest.mark.parametrize("curve", [1, 2])
def test_noalloc_matches_regular_two_calls(cuda_lib, curve):
    # every case twice in a row, then the next: each call reuses the array
    for n, inverse, coset, seed in CASES:
        x = kb().gen_scalars(curve, seed + curve, n)
        want = kb().ntt_fr(curve, x, inverse=inverse, coset=coset)
        for _ in range(2):
            assert kb().ntt_fr_noalloc(curve, x, inverse=inverse, coset=coset) == want, (n, inverse, coset)


def test_noalloc_warm_call_allocates_nothing(cuda_lib):
    """After one pass over every case (module loading and the per-device
    address lookup happen on first use), a second pass leaves the device's
    free memory exactly where it was."""
    import torch
    inputs = [(curve, kb().gen_scalars(curve, seed, n), inverse, coset)
              for curve in (1, 2) for n, inverse, coset, seed in CASES]
    for curve, x, inverse, coset in inputs:
        kb().ntt_fr_noalloc(curve, x, inverse=inverse, coset=coset)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for curve, x, inverse, coset in inputs:
        kb().ntt_fr_noalloc(curve, x, inverse=inverse, coset=coset)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_beyond_limit(cuda_lib):
    n = 1 << 17
    buf = ctypes.create_string_buffer(32)  # never read: the size check comes first
    assert kb().lib().ntt_fr_transform_noalloc(2, buf, n, 0, 0) == -2
    assert "2^16" in kb().last_error()
    assert kb().lib().ntt_fr_transform_noalloc(2, buf, 3, 0, 0) == -2
