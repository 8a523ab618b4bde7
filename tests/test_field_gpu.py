"""Field arithmetic on the device.  Products: the Karatsuba product and
squaring and the interleaved product against the oracle's CPU product
(kb200_field_mul_check).  Inversion: the binary-GCD inversion every kernel
uses against the Fermat chain a^(p-2), and x * x^-1 = 1
(kb200_field_inverse_check, edge values 0, 1, 2, p-1, p-2, (p-1)/2 and
seeded random elements)."""
from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("field", [0, 1, 2, 3])
def test_inverse_matches_fermat(cuda_lib, field):
    import crypto_b200
    bad = ctypes.c_ulonglong(1)
    rc = crypto_b200.lib().kb200_field_inverse_check(field, 1000 + field, 1 << 16, ctypes.byref(bad))
    assert rc == 0, crypto_b200.last_error()
    assert bad.value == 0


@pytest.mark.parametrize("field", [0, 1, 2, 3])
def test_products_match_oracle(cuda_lib, field):
    """The Karatsuba product and squaring every kernel calls, and the
    interleaved product kernels inline, against the oracle's CPU product
    (the reference's 64-bit-limb CIOS restated): edge operands 0, 1, p - 1,
    values with all-ones halves (the Karatsuba sums' carry bits), and
    seeded random elements below p."""
    import random

    import _oracle as O
    import crypto_b200
    p = {0: O.FP[2], 1: O.FR[2], 2: O.FP[1], 3: O.FR[1]}[field]
    nb = 48 if field == 0 else 32
    half = nb * 4  # bits per half
    rng = random.Random(field)
    edge = [0, 1, 2, p - 1, p - 2, (p - 1) // 2, (1 << half) - 1, p - 1 - ((1 << half) - 1),
            ((1 << (8 * nb)) - 1) % p, ((1 << half) - 1) << half]
    vals = [v % p for v in edge] + [rng.randrange(p) for _ in range(4000)]
    avals = vals + vals[::-1]
    bvals = vals[::-1] + vals
    n = len(avals)
    A = b"".join(v.to_bytes(nb, "little") for v in avals)
    B = b"".join(v.to_bytes(nb, "little") for v in bvals)
    om = ctypes.create_string_buffer(n * nb)
    osq = ctypes.create_string_buffer(n * nb)
    bad = ctypes.c_ulonglong(1)
    rc = crypto_b200.lib().kb200_field_mul_check(field, A, B, n, om, osq, ctypes.byref(bad))
    assert rc == 0, crypto_b200.last_error()
    assert bad.value == 0
    for i in range(n):
        a, b = A[nb * i:nb * (i + 1)], B[nb * i:nb * (i + 1)]
        assert om.raw[nb * i:nb * (i + 1)] == O.field_mul(field, a, b), i
        assert osq.raw[nb * i:nb * (i + 1)] == O.field_mul(field, a, a), i
