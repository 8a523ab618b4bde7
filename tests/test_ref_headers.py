"""A C caller written against the reference's own headers (c-abi/crypto.h,
gpukit/include/kinet/gpukit/multi_pippenger.h, bls/c-abi/c_bls_pairing.h)
compiles and links against libkinet_b200.so, and the library's header can sit
in the same translation unit (every shared declaration type-compatible).
tests/c/ref_headers_drop_in.c runs argument-check calls only, so no GPU is
needed.  Needs the reference tree (KINET_REFERENCE, default /root/reference);
skipped where it is absent."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("KINET_REFERENCE", "/root/reference"))
LIB = ROOT / "crypto_b200" / "_lib"


@pytest.mark.skipif(not (REF / "c-abi" / "crypto.h").exists(), reason="reference headers absent")
@pytest.mark.parametrize("both", [False, True])
def test_reference_headers_compile_link_run(tmp_path, both):
    import crypto_b200
    crypto_b200.lib()  # built
    src = ROOT / "tests" / "c" / "ref_headers_drop_in.c"
    inc = [f"-I{REF / 'c-abi'}", f"-I{REF / 'include'}", f"-I{REF / 'attestation' / 'include'}",
           f"-I{REF / 'gpukit' / 'include'}", f"-I{REF / 'bls' / 'c-abi'}", f"-I{ROOT / 'include'}"]
    objs = []
    for part in ("CRYPTO", "GPUKIT", "BLS", "MAIN"):
        obj = tmp_path / f"{part}.o"
        cmd = ["gcc", "-std=c11", "-Wall", "-Werror", f"-DPART_{part}", *inc, "-c", str(src), "-o", str(obj)]
        if both:
            cmd.insert(1, "-DKB200_BOTH_HEADERS")
        res = subprocess.run(cmd, capture_output=True, text=True)
        assert res.returncode == 0, res.stderr
        objs.append(str(obj))
    exe = tmp_path / "drop_in"
    res = subprocess.run(["gcc", "-o", str(exe), *objs, f"-L{LIB}", "-lkinet_b200", f"-Wl,-rpath,{LIB}"],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and "ok" in run.stdout, run.stdout + run.stderr
