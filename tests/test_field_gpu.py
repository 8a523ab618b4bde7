"""Field inversion on the device: the binary-GCD inversion every kernel uses
against the Fermat chain a^(p-2), and x * x^-1 = 1 (kb200_field_inverse_check,
edge values 0, 1, 2, p-1, p-2, (p-1)/2 and seeded random elements)."""
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
