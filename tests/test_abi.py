"""CPU-side checks of the C ABI: the library loads, exports every symbol its
header declares, validates arguments before touching a device, refuses to
run without a GPU (no CPU fallback), and the seeded input generator is
deterministic and canonical."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

import _oracle as O

ROOT = Path(__file__).resolve().parents[1]


def kb():
    import crypto_b200
    return crypto_b200


def declared_symbols() -> list[str]:
    names = []
    for h in (ROOT / "include").rglob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "defined"):
                names.append(name)
    return sorted(set(names))


def test_header_symbols_exported():
    L = kb().lib()
    names = declared_symbols()
    assert "gpukit_multi_pippenger" in names and "kzg_commit_fr" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_argument_checks_precede_device_use():
    k = kb()
    out = ctypes.create_string_buffer(96)
    assert k.msm_rc(2, None, None, 4, out) == -1
    assert k.msm_rc(2, b"\0" * 32, b"\0" * 96, 1, None) == -1
    assert k.msm_rc(0, b"\0" * 32, b"\0" * 64, 1, out) == -5
    assert k.msm_rc(17, b"\0" * 32, b"\0" * 64, 1, out) == -3
    L = k.lib()
    buf = ctypes.create_string_buffer(96)
    assert L.ntt_fr_forward(2, buf, 3, 0) == -2
    assert L.ntt_fr_forward(2, None, 4, 0) == -1
    assert L.kzg_commit_fr(None, 4, out) == -1


def test_no_cpu_fallback_without_gpu():
    k = kb()
    if k.device_available():
        pytest.skip("a GPU is present")
    out = ctypes.create_string_buffer(96)
    rc = k.msm_rc(2, b"\0" * 32, b"\0" * 96, 1, out)
    assert rc == -4                          # GPUKIT_ERR_DISPATCH, not a CPU result
    assert "CUDA" in k.last_error()
    buf = ctypes.create_string_buffer(bytes(64), 64)
    assert k.lib().ntt_fr_forward(2, buf, 2, 0) == -4


@pytest.mark.parametrize("curve", [1, 2])
def test_generator_deterministic_and_canonical(curve):
    a = kb().gen_scalars(curve, 42, 1000)
    b = kb().gen_scalars(curve, 42, 1000)
    c = kb().gen_scalars(curve, 43, 1000)
    assert a == b and a != c
    r = O.FR[curve]
    vals = [int.from_bytes(a[32 * i:32 * i + 32], "little") for i in range(1000)]
    assert all(v < r for v in vals)
    assert max(vals).bit_length() >= (254 if curve == 2 else 253)


def test_skewed_generator_mix():
    s = kb().gen_scalars(1, 7, 20000, kind=1)
    vals = [int.from_bytes(s[32 * i:32 * i + 32], "little") for i in range(20000)]
    zeros = sum(v == 0 for v in vals) / len(vals)
    ones = sum(v == 1 for v in vals) / len(vals)
    small = sum(1 < v < (1 << 64) for v in vals) / len(vals)
    assert 0.23 < zeros < 0.27 and 0.23 < ones < 0.27 and 0.18 < small < 0.22
    assert all(v < O.FR[1] for v in vals)


def test_window_planner():
    k = kb()
    # small MSMs use small windows, large MSMs large ones (more buckets)
    assert k.msm_window(2, 16) <= 6
    assert 14 <= k.msm_window(2, 1 << 22) <= 20
