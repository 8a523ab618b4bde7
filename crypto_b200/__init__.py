"""kinet-b200: B200-native polynomial-commitment path (Fr NTT, G1 MSM, KZG).

Thin Python binding over the C ABI in include/kinet_b200/crypto_b200.h.  The
compute lives in the CUDA library crypto_b200/_lib/libkinet_b200.so; this
module only marshals bytes.  There is no CPU fallback: loading fails loudly
if the library is missing, and every call reports the library's error code.

Wire formats (same as the reference's gpukit / crypto C ABI):
  scalar / Fr element : 32 bytes little-endian
  G1 point            : x || y big-endian (96 B BLS12-381, 64 B BN254),
                        all-zero = infinity
  compressed G1       : 48 bytes (BLS12-381)
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

CURVE_BN254 = 1
CURVE_BLS12_381 = 2
POINT_BYTES = {CURVE_BN254: 64, CURVE_BLS12_381: 96}

GPUKIT_OK = 0
CRYPTO_OK = 0

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libkinet_b200.so"
_lib: ctypes.CDLL | None = None


class KinetB200Error(RuntimeError):
    def __init__(self, fn: str, rc: int, msg: str):
        super().__init__(f"{fn} returned {rc}: {msg}")
        self.rc = rc


def lib() -> ctypes.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        path = os.environ.get("KINET_B200_LIB", str(_LIB_PATH))
        if not Path(path).exists():
            raise ImportError(f"kinet-b200 CUDA library not built: {path} "
                              "(run `python -m crypto_b200.build`)")
        L = ctypes.CDLL(path)
        c = ctypes
        sz, u8p, vp = c.c_size_t, c.c_char_p, c.c_void_p
        sigs = {
            "gpukit_multi_pippenger": (c.c_int, [c.c_uint32, u8p, u8p, sz, vp]),
            "gpukit_multi_pippenger_cuda": (c.c_int, [c.c_uint32, u8p, u8p, sz, vp]),
            "gpukit_multi_pippenger_subgroup": (c.c_int, [c.c_uint32, u8p, u8p, sz, vp]),
            "kb200_msm_device_subgroup": (c.c_int, [c.c_uint32, vp, vp, sz, vp, vp]),
            "kb200_msm_window_subgroup": (c.c_int, [c.c_uint32, sz]),
            "kb200_msm_entries_subgroup": (c.c_double, [c.c_uint32, sz]),
            "bls12_381_g1_msm": (c.c_int, [vp, vp, u8p, sz]),
            "kzg_blob_setup_load_g1_lagrange": (c.c_int, [u8p, sz]),
            "kzg_blob_setup_generate": (c.c_int, [u8p]),
            "kzg_blob_to_commit": (c.c_int, [u8p, vp]),
            "kzg_commit_to_proof": (c.c_int, [u8p, u8p, vp, vp]),
            "kb200_bls12_381_g1_msm_device": (c.c_int, [vp, sz, vp, vp, vp]),
            "ntt_forward": (c.c_int, [vp, sz, c.c_uint64, c.c_uint64]),
            "ntt_inverse": (c.c_int, [vp, sz, c.c_uint64, c.c_uint64]),
            "kb200_word_ntt_device": (c.c_int, [vp, vp, sz, c.c_uint64, c.c_uint64, c.c_int, vp]),
            "ntt_fr_forward": (c.c_int, [c.c_int, vp, sz, c.c_int]),
            "ntt_fr_inverse": (c.c_int, [c.c_int, vp, sz, c.c_int]),
            "ntt_fr_transform_noalloc": (c.c_int, [c.c_int, vp, sz, c.c_int, c.c_int]),
            "kzg_srs_load_g1": (c.c_int, [u8p, sz]),
            "kzg_srs_generate_g1": (c.c_int, [u8p, sz]),
            "kzg_srs_read_g1": (c.c_int, [vp, sz, sz]),
            "kzg_srs_size": (sz, []),
            "kzg_commit_fr": (c.c_int, [u8p, sz, vp]),
            "kzg_commit_batch": (c.c_int, [u8p, c.POINTER(sz), sz, vp]),
            "kb200_msm_device": (c.c_int, [c.c_uint32, vp, vp, sz, vp, vp]),
            "kb200_ntt_device": (c.c_int, [c.c_int, vp, sz, c.c_int, c.c_int, sz, vp]),
            "kb200_g1_fixed_base_device": (c.c_int, [c.c_uint32, vp, sz, vp, vp]),
            "kb200_fr_powers_device": (c.c_int, [c.c_int, vp, sz, vp, vp]),
            "kb200_kzg_commit_device": (c.c_int, [vp, sz, vp, vp]),
            "kb200_gen_scalars": (c.c_int, [c.c_int, c.c_uint64, sz, c.c_int, vp]),
            "kb200_last_error": (c.c_char_p, []),
            "kb200_device_available": (c.c_int, []),
            "kb200_msm_window": (c.c_int, [c.c_uint32, sz]),
            "kb200_msm_entries": (c.c_double, [c.c_uint32, sz]),
            "kb200_field_inverse_check": (c.c_int, [c.c_int, c.c_uint64, sz, c.POINTER(c.c_ulonglong)]),
            "kb200_field_mul_check": (c.c_int, [c.c_int, u8p, u8p, sz, vp, vp, c.POINTER(c.c_ulonglong)]),
            "kb200_launch_count": (c.c_ulonglong, []),
            "kzg_server_create": (vp, [sz, c.c_int, sz]),
            "kzg_server_submit": (c.c_int, [vp, u8p, sz, c.POINTER(c.c_uint64)]),
            "kzg_server_wait": (c.c_int, [vp, c.c_uint64, vp, c.POINTER(c.c_double), c.c_double]),
            "kzg_server_stats": (c.c_int, [vp, c.POINTER(c.c_double), c.POINTER(c.c_double),
                                           c.POINTER(c.c_double), c.POINTER(c.c_uint64), c.c_int]),
            "kzg_server_destroy": (c.c_int, [vp]),
            "kb200_autotune": (c.c_int, [c.c_uint32, c.c_int, c.c_int, c.c_char_p]),
            "kb200_autotune_load": (c.c_int, [c.c_char_p]),
            "kb200_tune_get": (c.c_int, [c.c_int, c.c_uint32, c.c_int]),
            "kb200_tune_set": (None, [c.c_int, c.c_uint32, c.c_int, c.c_int]),
            "kb200_profile_enable": (None, [c.c_int]),
            "kb200_msm_stage_ms": (c.c_int, [c.c_uint32, c.POINTER(c.c_float), c.c_int]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(fn: str, rc: int) -> None:
    if rc != 0:
        raise KinetB200Error(fn, rc, lib().kb200_last_error().decode(errors="replace"))


def last_error() -> str:
    return lib().kb200_last_error().decode(errors="replace")


def device_available() -> bool:
    return bool(lib().kb200_device_available())


# ---- MSM --------------------------------------------------------------------

def gpukit_multi_pippenger(curve: int, scalars: bytes, points: bytes, n: int) -> bytes:
    """sum_i scalars[i] * points[i]; mirrors gpukit_multi_pippenger."""
    out = ctypes.create_string_buffer(POINT_BYTES.get(curve, 96))
    _check("gpukit_multi_pippenger",
           lib().gpukit_multi_pippenger(curve, scalars, points, n, out))
    return out.raw


def gpukit_multi_pippenger_subgroup(curve: int, scalars: bytes, points: bytes, n: int) -> bytes:
    """The same sum for points the caller knows to lie in G1 (GLV split on
    BLS12-381); unspecified for BLS12-381 curve points outside G1."""
    out = ctypes.create_string_buffer(POINT_BYTES.get(curve, 96))
    _check("gpukit_multi_pippenger_subgroup",
           lib().gpukit_multi_pippenger_subgroup(curve, scalars, points, n, out))
    return out.raw


def bls12_381_g1_msm(xycs: bytes):
    """EIP-2537 BLS12_G1MSM: returns (status, rx || ry) with status 1 = ok,
    0 = invalid input, < 0 = backend error."""
    rx = ctypes.create_string_buffer(64)
    ry = ctypes.create_string_buffer(64)
    rc = lib().bls12_381_g1_msm(rx, ry, xycs, len(xycs))
    return rc, rx.raw + ry.raw


def kzg_blob_to_commit(blob: bytes):
    """(status, 48-byte commitment) for a 131072-byte blob."""
    out = ctypes.create_string_buffer(48)
    rc = lib().kzg_blob_to_commit(blob, out)
    return rc, out.raw


def kzg_commit_to_proof(blob: bytes, z: bytes):
    """(status, 48-byte proof, 32-byte big-endian y)."""
    proof = ctypes.create_string_buffer(48)
    y = ctypes.create_string_buffer(32)
    rc = lib().kzg_commit_to_proof(blob, z, proof, y)
    return rc, proof.raw, y.raw


def msm_rc(curve: int, scalars, points, n: int, out) -> int:
    """Raw call returning the status code (for error-behaviour tests)."""
    return lib().gpukit_multi_pippenger(curve, scalars, points, n, out)


# ---- NTT --------------------------------------------------------------------

def word_ntt_rc(words, n: int, modulus: int, root: int, inverse: bool = False) -> int:
    """ntt_forward / ntt_inverse in place on a writable buffer of uint64
    words (a numpy array or ctypes buffer); returns the status code."""
    ptr = words.ctypes.data if hasattr(words, "ctypes") else ctypes.addressof(words)
    fn = lib().ntt_inverse if inverse else lib().ntt_forward
    return fn(ptr, n, modulus, root)


def word_ntt(words, modulus: int, root: int, inverse: bool = False):
    """Word-prime NTT of a uint64 numpy array (returns a transformed copy)."""
    import numpy as np
    a = np.ascontiguousarray(np.array(words, dtype=np.uint64))
    _check("ntt_inverse" if inverse else "ntt_forward",
           word_ntt_rc(a, len(a), modulus, root, inverse))
    return a


def ntt_fr(curve: int, data: bytes, inverse: bool = False, coset: bool = False) -> bytes:
    n = len(data) // 32
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    fn = lib().ntt_fr_inverse if inverse else lib().ntt_fr_forward
    _check("ntt_fr_inverse" if inverse else "ntt_fr_forward", fn(curve, buf, n, int(coset)))
    return buf.raw


def ntt_fr_noalloc(curve: int, data: bytes, inverse: bool = False, coset: bool = False) -> bytes:
    """Allocation-free variant (n <= 2^16), scratch in a static device array."""
    n = len(data) // 32
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    _check("ntt_fr_transform_noalloc",
           lib().ntt_fr_transform_noalloc(curve, buf, n, int(inverse), int(coset)))
    return buf.raw


# ---- KZG --------------------------------------------------------------------

def kzg_srs_generate(tau: bytes, n: int) -> None:
    _check("kzg_srs_generate_g1", lib().kzg_srs_generate_g1(tau, n))


def kzg_srs_load(points: bytes) -> None:
    _check("kzg_srs_load_g1", lib().kzg_srs_load_g1(points, len(points) // 96))


def kzg_srs_read(offset: int, count: int) -> bytes:
    out = ctypes.create_string_buffer(96 * count)
    _check("kzg_srs_read_g1", lib().kzg_srs_read_g1(out, offset, count))
    return out.raw


def kzg_srs_size() -> int:
    return int(lib().kzg_srs_size())


def kzg_commit(evals: bytes) -> bytes:
    out = ctypes.create_string_buffer(48)
    _check("kzg_commit_fr", lib().kzg_commit_fr(evals, len(evals) // 32, out))
    return out.raw


def kzg_commit_batch(evals: bytes, sizes: list[int]) -> list[bytes]:
    arr = (ctypes.c_size_t * len(sizes))(*sizes)
    out = ctypes.create_string_buffer(48 * len(sizes))
    _check("kzg_commit_batch", lib().kzg_commit_batch(evals, arr, len(sizes), out))
    return [out.raw[48 * i:48 * i + 48] for i in range(len(sizes))]


# ---- inputs -----------------------------------------------------------------

def gen_scalars(curve: int, seed: int, n: int, kind: int = 0) -> bytes:
    """Seeded xorshift64* Fr scalars (kind 0 uniform, 1 skewed)."""
    out = ctypes.create_string_buffer(32 * n)
    _check("kb200_gen_scalars", lib().kb200_gen_scalars(curve, seed, n, kind, out))
    return out.raw


def msm_window(curve: int, n: int, subgroup: bool = False) -> int:
    f = lib().kb200_msm_window_subgroup if subgroup else lib().kb200_msm_window
    return int(f(curve, n))


def launch_count() -> int:
    """Kernel launches issued by this library since it was loaded."""
    return int(lib().kb200_launch_count())


def profile_enable(on: bool) -> None:
    lib().kb200_profile_enable(int(on))


MSM_STAGES = ("wire_to_table", "recode", "sort", "pair", "accumulate", "fold", "reduce", "combine")


def msm_stage_ms(curve: int) -> dict[str, float]:
    buf = (ctypes.c_float * 16)()
    k = lib().kb200_msm_stage_ms(curve, buf, 16)
    return {MSM_STAGES[i]: float(buf[i]) for i in range(max(k, 0))}


# ---- serving ------------------------------------------------------------------

class KzgServer:
    """Continuous-batching commit server over the resident SRS (C ABI
    kzg_server_*).  submit() returns a ticket; wait() returns (commit, ms)."""

    def __init__(self, max_batch: int = 64, slots: int = 2, mem_budget: int = 0):
        self.h = lib().kzg_server_create(max_batch, slots, mem_budget)
        if not self.h:
            raise KinetB200Error("kzg_server_create", -4, last_error())

    def submit(self, evals: bytes) -> int:
        t = ctypes.c_uint64()
        _check("kzg_server_submit", lib().kzg_server_submit(self.h, evals, len(evals) // 32,
                                                            ctypes.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0):
        out = ctypes.create_string_buffer(48)
        lat = ctypes.c_double()
        rc = lib().kzg_server_wait(self.h, ticket, out, ctypes.byref(lat), timeout_ms)
        if rc == 1:
            return None
        _check("kzg_server_wait", rc)
        return out.raw, lat.value

    def stats(self, reset: bool = False) -> dict:
        p50, p99, cps = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        done = ctypes.c_uint64()
        _check("kzg_server_stats", lib().kzg_server_stats(self.h, ctypes.byref(p50), ctypes.byref(p99),
                                                          ctypes.byref(cps), ctypes.byref(done), int(reset)))
        return {"p50_ms": p50.value, "p99_ms": p99.value, "commits_per_s": cps.value,
                "completed": done.value}

    def close(self) -> None:
        if self.h:
            lib().kzg_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
