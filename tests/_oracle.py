"""ctypes wrappers for the CPU checker (oracle/).  Test infrastructure only.

  orc  -> oracle/_build/liboracle.so   (C restatement of the reference path)
  ref  -> oracle/_ref/libref_msm.so    (the reference's own CPU MSM, built
                                        unmodified from its sources)
  ref_ntt -> oracle/_ref/libref_ntt.so (the reference's word-prime NTT and its
                                        C-ABI shim, built unmodified)
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
ORC_PATH = ROOT / "oracle" / "_build" / "liboracle.so"
REF_PATH = ROOT / "oracle" / "_ref" / "libref_msm.so"
REF_NTT_PATH = ROOT / "oracle" / "_ref" / "libref_ntt.so"

_orc = None
_ref = None
_ref_ntt = None


def orc() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        if not ORC_PATH.exists():
            subprocess.run(["make", "-C", str(ROOT / "oracle"), "all"], check=True,
                           capture_output=True)
        L = ctypes.CDLL(str(ORC_PATH))
        sz = ctypes.c_size_t
        for name, args in {
            "orc_msm": [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, sz, ctypes.c_void_p],
            "orc_msm_naive": [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, sz, ctypes.c_void_p],
            "orc_g1_mul_gen": [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_void_p],
            "orc_g1_mul": [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p],
            "orc_g1_add": [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p],
            "orc_g1_on_curve": [ctypes.c_uint32, ctypes.c_char_p],
            "orc_ntt": [ctypes.c_uint32, ctypes.c_void_p, sz, ctypes.c_int, ctypes.c_int],
            "orc_dft": [ctypes.c_uint32, ctypes.c_void_p, sz, ctypes.c_int, ctypes.c_int],
            "orc_root_of_unity": [ctypes.c_uint32, sz, ctypes.c_void_p],
            "orc_g1_compress": [ctypes.c_char_p, ctypes.c_void_p],
            "orc_kzg_commit": [ctypes.c_char_p, sz, ctypes.c_char_p, ctypes.c_void_p],
            "orc_fr_powers": [ctypes.c_uint32, ctypes.c_char_p, sz, ctypes.c_void_p],
            "orc_field_mul": [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p],
            "orc_field_inv": [ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p],
            "orc_bls12_381_g1_msm": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, sz],
            "orc_kzg_blob_commit": [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p],
            "orc_kzg_blob_proof": [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p,
                                   ctypes.c_void_p],
            "orc_word_ntt_forward": [ctypes.c_void_p, sz, ctypes.c_uint64, ctypes.c_uint64],
            "orc_word_ntt_inverse": [ctypes.c_void_p, sz, ctypes.c_uint64, ctypes.c_uint64],
            "orc_gen_scalars": [ctypes.c_uint32, ctypes.c_uint64, sz, ctypes.c_int, ctypes.c_void_p],
            "orc_g1_fixed_base_batch": [ctypes.c_uint32, ctypes.c_void_p, sz, ctypes.c_void_p,
                                        ctypes.c_int],
        }.items():
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = args
        _orc = L
    return _orc


def gen_scalars(curve: int, seed: int, n: int, kind: int = 0) -> bytes:
    """The library's seeded scalar streams (kb200_gen_scalars), made on the CPU."""
    out = ctypes.create_string_buffer(32 * n)
    assert orc().orc_gen_scalars(curve, seed, n, kind, out) == 0
    return out.raw


def fixed_base_points(curve: int, scalars: bytes, threads: int = 0) -> bytes:
    """k_i * G for every 32-byte LE scalar k_i (CPU, fixed-base windows)."""
    import os
    n = len(scalars) // 32
    out = ctypes.create_string_buffer(PB[curve] * n)
    src = ctypes.create_string_buffer(bytes(scalars), len(scalars))
    rc = orc().orc_g1_fixed_base_batch(curve, src, n, out, threads or (os.cpu_count() or 1))
    assert rc == 0, rc
    return out.raw


def ref_available() -> bool:
    return REF_PATH.exists()


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        L = ctypes.CDLL(str(REF_PATH))
        sz = ctypes.c_size_t
        L.ref_msm.restype = ctypes.c_int
        L.ref_msm.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, sz, ctypes.c_void_p]
        L.ref_msm_parallel.restype = ctypes.c_int
        L.ref_msm_parallel.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, sz,
                                       ctypes.c_void_p, ctypes.c_int]
        L.ref_g1_mul_gen.restype = ctypes.c_int
        L.ref_g1_mul_gen.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_void_p]
        _ref = L
    return _ref


PB = {1: 64, 2: 96}


def msm(curve: int, scalars: bytes, points: bytes, n: int) -> bytes:
    out = ctypes.create_string_buffer(PB[curve])
    rc = orc().orc_msm(curve, scalars, points, n, out)
    assert rc == 0, rc
    return out.raw


def msm_naive(curve: int, scalars: bytes, points: bytes, n: int) -> bytes:
    out = ctypes.create_string_buffer(PB[curve])
    assert orc().orc_msm_naive(curve, scalars, points, n, out) == 0
    return out.raw


def ref_msm(curve: int, scalars: bytes, points: bytes, n: int, threads: int = 1) -> bytes:
    out = ctypes.create_string_buffer(PB[curve])
    if threads <= 1:
        rc = ref().ref_msm(curve, scalars, points, n, out)
    else:
        rc = ref().ref_msm_parallel(curve, scalars, points, n, out, threads)
    assert rc == 0, rc
    return out.raw


def g1_mul_gen(curve: int, k: int) -> bytes:
    out = ctypes.create_string_buffer(PB[curve])
    assert orc().orc_g1_mul_gen(curve, k.to_bytes(32, "little"), out) == 0
    return out.raw


def g1_mul(curve: int, point: bytes, k: int) -> bytes:
    out = ctypes.create_string_buffer(PB[curve])
    assert orc().orc_g1_mul(curve, point, k.to_bytes(32, "little"), out) == 0
    return out.raw


def g1_add(curve: int, p: bytes, q: bytes) -> bytes:
    out = ctypes.create_string_buffer(PB[curve])
    assert orc().orc_g1_add(curve, p, q, out) == 0
    return out.raw


def on_curve(curve: int, p: bytes) -> bool:
    return orc().orc_g1_on_curve(curve, p) == 1


def ntt(curve: int, data: bytes, inverse: bool = False, coset: bool = False) -> bytes:
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    rc = orc().orc_ntt(curve, buf, len(data) // 32, int(inverse), int(coset))
    assert rc == 0, rc
    return buf.raw


def dft(curve: int, data: bytes, inverse: bool = False, coset: bool = False) -> bytes:
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    assert orc().orc_dft(curve, buf, len(data) // 32, int(inverse), int(coset)) == 0
    return buf.raw


def compress(point96: bytes) -> bytes:
    out = ctypes.create_string_buffer(48)
    assert orc().orc_g1_compress(point96, out) == 0
    return out.raw


def kzg_commit(evals: bytes, srs: bytes) -> bytes:
    out = ctypes.create_string_buffer(48)
    rc = orc().orc_kzg_commit(evals, len(evals) // 32, srs, out)
    assert rc == 0, rc
    return out.raw


def fr_powers(curve: int, tau: bytes, n: int) -> bytes:
    out = ctypes.create_string_buffer(32 * n)
    assert orc().orc_fr_powers(curve, tau, n, out) == 0
    return out.raw


def bls12_381_g1_msm(xycs: bytes):
    """Oracle EIP-2537 G1 MSM: (status 1/0, rx || ry)."""
    rx = ctypes.create_string_buffer(64)
    ry = ctypes.create_string_buffer(64)
    rc = orc().orc_bls12_381_g1_msm(rx, ry, xycs, len(xycs))
    return rc, rx.raw + ry.raw


def kzg_blob_commit(blob: bytes, srs: bytes):
    out = ctypes.create_string_buffer(48)
    rc = orc().orc_kzg_blob_commit(blob, srs, out)
    return rc, out.raw


def kzg_blob_proof(blob: bytes, z: bytes, srs: bytes):
    proof = ctypes.create_string_buffer(48)
    y = ctypes.create_string_buffer(32)
    rc = orc().orc_kzg_blob_proof(blob, z, srs, proof, y)
    return rc, proof.raw, y.raw


def word_ntt(words, q: int, root: int, inverse: bool = False):
    """Oracle word-prime NTT (ntt_forward / ntt_inverse contract) of a uint64
    numpy array; returns (status, transformed copy)."""
    import numpy as np
    a = np.array(words, dtype=np.uint64)
    f = orc().orc_word_ntt_inverse if inverse else orc().orc_word_ntt_forward
    return f(a.ctypes.data, len(a), q, root), a


def ref_ntt_available() -> bool:
    return REF_NTT_PATH.exists()


def ref_word_ntt(a, n: int, q: int, root: int, inverse: bool = False) -> int:
    """The reference's own ntt_forward / ntt_inverse, in place on a uint64
    numpy array."""
    global _ref_ntt
    if _ref_ntt is None:
        L = ctypes.CDLL(str(REF_NTT_PATH))
        for name in ("ntt_forward", "ntt_inverse"):
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64]
        _ref_ntt = L
    f = _ref_ntt.ntt_inverse if inverse else _ref_ntt.ntt_forward
    return f(a.ctypes.data, n, q, root)


# Field moduli for host-side checks (canonical integers).
FR = {2: 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001,
      1: 21888242871839275222246405745257275088548364400416034343698204186575808495617}
FP = {2: 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB,
      1: 21888242871839275222246405745257275088696311157297823662689037894645226208583}


def field_mul(which: int, a: bytes, b: bytes) -> bytes:
    """Canonical a * b in field `which` (0 BLS12-381 Fp, 1 BLS12-381 Fr,
    2 BN254 Fp, 3 BN254 Fr), little-endian bytes of the field's width."""
    out = ctypes.create_string_buffer(len(a))
    assert orc().orc_field_mul(which, a, b, out) == 0
    return out.raw
