"""Builds the kinet-b200 shared library in-tree with nvcc for sm_100a.

    python -m crypto_b200.build            # incremental
    python -m crypto_b200.build --force    # rebuild everything

Each translation unit is compiled separately (in parallel) into
crypto_b200/_build/, then linked into crypto_b200/_lib/libkinet_b200.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc"
OBJ = HERE / "_build"
LIB = HERE / "_lib" / "libkinet_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
HOSTFLAGS = ["-O2", "-std=c++17", "-fPIC"]

SOURCES = ["msm.cu", "msm_bls.cu", "msm_bn.cu", "ntt.cu", "kzg.cu", "scan.cu", "capi.cu", "batch.cu", "serve.cu", "autotune.cu", "wntt.cu", "eip2537.cu", "kzg_blob.cu", "selfcheck.cu",
           "inputs.cpp"]


def _headers() -> list[Path]:
    return sorted(SRC.glob("*.cuh")) + sorted((HERE.parent / "include").rglob("*.h"))


def _compile(src: Path, force: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if not force and obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    if src.suffix == ".cu":
        cmd = [NVCC, *CUFLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [NVCC, "-x", "c++", "-Xcompiler", " ".join(HOSTFLAGS), "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if "spill" in res.stderr and "0 bytes spill" not in res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    srcs = [SRC / s for s in SOURCES if (SRC / s).exists()]
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    print(build(a.force, a.j))
