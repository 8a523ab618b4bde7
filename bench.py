"""Benchmark: BLS12-381 G1 MSM at n = 2^22 (the headline), one GPU per rank.

A step is one full MSM (sum of 2^22 scalar * point products, uniform Fr
scalars, points s_i * G1 with seeded s_i) with inputs resident in HBM.
Inputs are 512 MiB (> 126 MB L2), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is Mpts/s over all ranks (each rank
runs its own independent MSM: replicas, weak scaling).  `e2e` is the same
metric through the drop-in C ABI (gpukit_multi_pippenger) from pinned host
buffers, host<->device copies included.  `--impl reference` times the
reference's own CPU MSM (gpukit_multi_pippenger_cpu, built from its sources
into oracle/_ref) on all host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CURVE = 2
LOGN = 22
PB = 96
N_LIMBS = 12
SM_COUNT = 148
IMAD_PER_CLK_SM = 64
# The headline workload's seeds: scalars s_i from stream 1, points k_i * G1
# with k_i from stream 1001 (uniform Fr, xorshift64* with rejection).
SCALAR_SEED = 1
POINT_SEED = 1001
# One step of the reference arm: a 2^20-point quarter of the 2^22 workload.
REF_BLOCK_LOG = 20
GOLDEN_LARGE = ROOT / "tests" / "golden" / "large.json"


def headline_config(logn: int) -> dict:
    """The workload both arms time (identical in both JSON lines)."""
    return {"workload": f"BLS12-381 G1 MSM n=2^{logn}: sum of s_i * P_i, s_i uniform Fr "
                        f"(seed {SCALAR_SEED}), P_i = k_i * G1 with k_i uniform Fr (seed {POINT_SEED})",
            "curve": "BLS12-381", "n": 1 << logn}


def golden_expected(logn: int):
    """Expected sum (hex) of the headline workload at 2^logn (its seeds), from
    the reference CPU MSM, or None when no golden case holds that workload."""
    if not GOLDEN_LARGE.exists():
        return None
    for c in json.loads(GOLDEN_LARGE.read_text())["msm"]:
        if (c["curve"], c["log_n"], c["kind"], c["scalar_seed"], c["point_seed"]) == \
                (CURVE, logn, 0, SCALAR_SEED, POINT_SEED):
            return c["expected"]
    return None


def mont_imad(nlimbs: int) -> int:
    return 4 * nlimbs * nlimbs + nlimbs


def w_msm(n: int, nlimbs: int) -> int:
    """Algorithmic IMAD of an MSM: 6 Montgomery products per bucket addition
    (batch-affine), min over c in [4,16] of ceil(256/c) * (n + 2^c)."""
    best = min(((256 + c - 1) // c) * (n + (1 << c)) for c in range(4, 17))
    return 6 * mont_imad(nlimbs) * best


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        # the sampler must be running before the timed region starts: wait for
        # its first row (nvidia-smi takes a few hundred ms to start)
        self.first_rows = 0
        deadline = time.time() + 5.0
        while self.proc and time.time() < deadline:
            with open(self.path) as f:
                self.first_rows = sum(1 for line in f if line.count(",") >= 7)
            if self.first_rows:
                break
            time.sleep(0.02)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        lines = [line for line in open(self.path) if line.count(",") >= 7]
        # rows written during the timed region; if it was too short for one,
        # the row taken just before it
        during = lines[self.first_rows:] or lines[max(0, self.first_rows - 1):self.first_rows]
        for line in during:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[4:8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows),
                "samples_in_timed_region": len(lines) - self.first_rows}


def setup_dist():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:  # host-side rank logic without a GPU (tests)
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    else:
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v: float) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def ref_threads() -> int:
    """Host threads for the reference CPU MSM: all cores, at most 16, so each
    slice of a 2^20-point step keeps >= 2^16 points and the reference picks
    the 12-bit window it uses for the whole 2^22 call."""
    return max(1, min(os.cpu_count() or 1, 16))


def cpu_workload(n: int):
    """The headline workload built on the CPU by the oracle's restated input
    generators (no GPU and no CUDA library involved)."""
    import _oracle as O
    scs = O.gen_scalars(CURVE, SCALAR_SEED, n)
    pts = O.fixed_base_points(CURVE, O.gen_scalars(CURVE, POINT_SEED, n))
    return scs, pts


def ref_block(scs: bytes, pts: bytes, n: int, block: int, threads: int):
    """The reference's own gpukit_multi_pippenger_cpu on one 2^REF_BLOCK_LOG
    block of the workload, split into `threads` contiguous slices run in
    parallel and summed with the reference g1_add.  Returns (seconds, sum)."""
    import _oracle as O
    m = min(n, 1 << REF_BLOCK_LOG)
    lo = (block * m) % n
    out = ctypes.create_string_buffer(PB)
    t0 = time.perf_counter()
    rc = O.ref().ref_msm_parallel(CURVE, scs[32 * lo:32 * (lo + m)], pts[PB * lo:PB * (lo + m)], m,
                                  out, threads)
    dt = time.perf_counter() - t0
    assert rc == 0, rc
    return dt, out.raw


def ref_sample_text(n: int, threads: int) -> str:
    m = min(n, 1 << REF_BLOCK_LOG)
    return (f"each step: the reference gpukit_multi_pippenger_cpu (built unmodified from its sources) on "
            f"one 2^{m.bit_length() - 1}-point block of the 2^{n.bit_length() - 1} workload (blocks in turn), "
            f"split into {threads} contiguous slices of {m // threads} points on {threads} threads and "
            f"summed with the reference g1_add; the slices use the 12-bit window the reference "
            f"picks for the whole call (its bucket overhead per point is 2^12/{m // threads} against "
            f"2^12/2^{n.bit_length() - 1})")


def make_inputs(n: int, seed: int):
    """Seeded uniform Fr scalars and points s_i * G1 (s_i seeded), on device."""
    import torch
    import crypto_b200 as kb
    sc = kb.gen_scalars(CURVE, seed, n)
    ks = kb.gen_scalars(CURVE, seed + POINT_SEED - SCALAR_SEED, n)
    d_sc = torch.frombuffer(bytearray(sc), dtype=torch.uint8).cuda()
    d_ks = torch.frombuffer(bytearray(ks), dtype=torch.uint8).cuda()
    d_pts = torch.empty(n * PB, dtype=torch.uint8, device="cuda")
    rc = kb.lib().kb200_g1_fixed_base_device(CURVE, d_ks.data_ptr(), n, d_pts.data_ptr(),
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, kb.last_error()
    torch.cuda.synchronize()
    del d_ks
    return d_sc, d_pts


def w_ntt(n: int) -> int:
    """Algorithmic IMAD of one Fr NTT: (n/2) log2 n Montgomery products, M(8) each."""
    return (n // 2) * (n.bit_length() - 1) * mont_imad(8)


def time_device(fn, steps: int, warmup: int) -> float:
    """Mean ms per call of fn (queued on torch's current stream), CUDA events."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def bench_extra(args, peak_imad: float) -> dict:
    """The other single-transform configurations: BLS12-381 MSM 2^20, BN254 MSM
    2^24 (uniform and skewed scalars), BLS12-381 Fr NTT 2^24 forward + inverse,
    BN254 coset NTT 2^26 forward + inverse, word-prime NTT 2^20 (Goldilocks and
    Cyclone-FFT primes), the EIP-2537 G1 MSM at 2^16 entries and the EIP-4844
    blob commitment and proof.  Device-resident inputs unless a case says
    otherwise."""
    import torch
    import crypto_b200 as kb
    L = kb.lib()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {}

    def msm_case(curve, logn, kind, label):
        n = 1 << logn
        pb = 96 if curve == 2 else 64
        sc = kb.gen_scalars(curve, 31 + logn, n, kind)
        ks = kb.gen_scalars(curve, 77 + logn, n)
        d_sc = torch.frombuffer(bytearray(sc), dtype=torch.uint8).cuda()
        d_ks = torch.frombuffer(bytearray(ks), dtype=torch.uint8).cuda()
        d_pts = torch.empty(n * pb, dtype=torch.uint8, device="cuda")
        assert L.kb200_g1_fixed_base_device(curve, d_ks.data_ptr(), n, d_pts.data_ptr(), sp) == 0
        del d_ks
        d_out = torch.empty(pb, dtype=torch.uint8, device="cuda")
        kb.profile_enable(True)
        ms = time_device(lambda: L.kb200_msm_device(curve, d_sc.data_ptr(), d_pts.data_ptr(), n,
                                                     d_out.data_ptr(), sp), 3, 2)
        stage = kb.msm_stage_ms(curve)
        kb.profile_enable(False)
        nl = 12 if curve == 2 else 8
        out[label] = {"n": n, "ms": ms, "mpts_per_s": n / ms / 1e3, "window_bits": kb.msm_window(curve, n),
                      "imad_frac": w_msm(n, nl) / (ms / 1e3) / peak_imad, "stage_ms": stage}
        del d_sc, d_pts, d_out
        torch.cuda.empty_cache()

    def ntt_case(curve, logn, coset, label):
        n = 1 << logn
        x = kb.gen_scalars(curve, 5 + logn, n)
        d = torch.frombuffer(bytearray(x), dtype=torch.uint8).cuda()

        def fwd_inv():
            assert L.kb200_ntt_device(curve, d.data_ptr(), n, 0, coset, 1, sp) == 0
            assert L.kb200_ntt_device(curve, d.data_ptr(), n, 1, coset, 1, sp) == 0

        ms = time_device(fwd_inv, 3, 2)
        assert d.cpu().numpy().tobytes() == x, "NTT round trip changed the data"
        passes = 1 if logn <= 12 else (2 if logn <= 20 else 3)
        bytes_moved = 2 * passes * 64 * n + 2 * (passes - 1) * 32 * n
        out[label] = {"n": n, "coset": bool(coset), "ms_fwd_plus_inv": ms,
                      "imad_frac": 2 * w_ntt(n) / (ms / 1e3) / peak_imad,
                      "hbm_gbs": bytes_moved / (ms / 1e3) / 1e9}
        del d
        torch.cuda.empty_cache()

    def word_ntt_case(q, g, logn, label):
        """ntt_forward on the six-step path (2^16 < n <= 2^20): device time
        of forward + inverse on resident words, the host-buffer C-ABI call,
        and the reference's own CPU body on the same input."""
        import numpy as np
        n = 1 << logn
        root = pow(g, (q - 1) // (2 * n), q)
        root_inv = pow(root, q - 2, q)
        x = np.random.Generator(np.random.PCG64(logn)).bit_generator.random_raw(n).astype(np.uint64) % np.uint64(q)
        d = torch.from_numpy(x.view(np.int64).copy()).cuda()

        def fwd_inv():
            assert L.kb200_word_ntt_device(d.data_ptr(), None, n, q, root, 0, sp) == 0
            assert L.kb200_word_ntt_device(d.data_ptr(), None, n, q, root_inv, 1, sp) == 0

        ms = time_device(fwd_inv, 3, 5)
        assert np.array_equal(d.cpu().numpy().view(np.uint64), x), "word NTT round trip changed the data"
        h = x.copy()
        assert L.ntt_forward(h.ctypes.data, n, q, root) == 0
        reps = 5
        t0 = time.perf_counter()
        for _ in range(reps):
            h[:] = x
            assert L.ntt_forward(h.ctypes.data, n, q, root) == 0
        e2e_ms = (time.perf_counter() - t0) * 1e3 / reps
        rec = {"n": n, "q": q, "ms_fwd_plus_inv_device": ms, "e2e_ms_forward": e2e_ms,
               "api": "ntt_forward (host words, copies included)"}
        ref = ROOT / "oracle" / "_ref" / "libref_ntt.so"
        if ref.exists():
            R = ctypes.CDLL(str(ref))
            R.ntt_forward.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64]
            g_ = x.copy()
            R.ntt_forward(g_.ctypes.data, n, q, root)  # builds its cached context
            g_[:] = x
            t0 = time.perf_counter()
            R.ntt_forward(g_.ctypes.data, n, q, root)
            rec["reference_cpu_ms_forward"] = (time.perf_counter() - t0) * 1e3
            rec["reference_cpu"] = "ntt_forward of the reference (ntt_large.cpp), 1 core"
            assert np.array_equal(g_, h), "GPU and reference outputs differ"
        out[label] = rec
        del d
        torch.cuda.empty_cache()

    def eip2537_case(logn, label):
        """bls12_381_g1_msm (EIP-2537 input: 160-byte entries, all checks)
        through the host C ABI, against the plain MSM of the same points."""
        import numpy as np
        n = 1 << logn
        ks = kb.gen_scalars(2, 91 + logn, n)
        d_ks = torch.frombuffer(bytearray(ks), dtype=torch.uint8).cuda()
        d_pts = torch.empty(n * 96, dtype=torch.uint8, device="cuda")
        assert L.kb200_g1_fixed_base_device(2, d_ks.data_ptr(), n, d_pts.data_ptr(), sp) == 0
        pts = d_pts.cpu().numpy().reshape(n, 96)
        sc = np.frombuffer(kb.gen_scalars(2, 92 + logn, n), dtype=np.uint8).reshape(n, 32)
        ent = np.zeros((n, 160), dtype=np.uint8)
        ent[:, 16:64] = pts[:, :48]
        ent[:, 80:128] = pts[:, 48:]
        ent[:, 128:] = sc[:, ::-1]  # little-endian scalars -> big-endian
        xycs = ent.tobytes()
        rx = ctypes.create_string_buffer(64)
        ry = ctypes.create_string_buffer(64)
        assert L.bls12_381_g1_msm(rx, ry, xycs, len(xycs)) == 1
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            assert L.bls12_381_g1_msm(rx, ry, xycs, len(xycs)) == 1
        ms = (time.perf_counter() - t0) * 1e3 / reps
        want = kb.gpukit_multi_pippenger(2, sc.tobytes(), pts.tobytes(), n)
        assert rx.raw[16:] + ry.raw[16:] == want, "EIP-2537 MSM differs from the plain MSM"
        out[label] = {"n": n, "e2e_ms": ms, "mpts_per_s": n / ms / 1e3,
                      "api": "bls12_381_g1_msm (host entries; range, curve and G1 checks included)"}
        del d_ks, d_pts
        torch.cuda.empty_cache()

    def blob_case(label):
        """kzg_blob_to_commit and kzg_commit_to_proof on one 4096-element blob
        over a resident test setup (host C ABI, copies included)."""
        import random
        r = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
        rng = random.Random(9)
        assert L.kzg_blob_setup_generate((12345).to_bytes(32, "little")) == 0
        blob = b"".join(rng.randrange(r).to_bytes(32, "big") for _ in range(4096))
        z = rng.randrange(r).to_bytes(32, "big")
        c = ctypes.create_string_buffer(48)
        pr = ctypes.create_string_buffer(48)
        y = ctypes.create_string_buffer(32)
        assert L.kzg_blob_to_commit(blob, c) == 0 and L.kzg_commit_to_proof(blob, z, pr, y) == 0
        reps = 20
        t0 = time.perf_counter()
        for _ in range(reps):
            assert L.kzg_blob_to_commit(blob, c) == 0
        commit_ms = (time.perf_counter() - t0) * 1e3 / reps
        t0 = time.perf_counter()
        for _ in range(reps):
            assert L.kzg_commit_to_proof(blob, z, pr, y) == 0
        proof_ms = (time.perf_counter() - t0) * 1e3 / reps
        out[label] = {"blob_to_commit_ms": commit_ms, "commit_to_proof_ms": proof_ms,
                      "api": "kzg_blob_to_commit / kzg_commit_to_proof (host, synchronous)"}

    msm_case(2, 20, 0, "msm_bls12_381_2^20")
    msm_case(1, 24, 0, "msm_bn254_2^24_uniform")
    msm_case(1, 24, 1, "msm_bn254_2^24_skewed")
    ntt_case(2, 24, 0, "ntt_bls12_381_2^24")
    ntt_case(1, 26, 1, "ntt_bn254_2^26_coset")
    word_ntt_case(0xFFFFFFFF00000001, 7, 20, "word_ntt_goldilocks_2^20")
    word_ntt_case(998244353, 3, 20, "word_ntt_cyclone_2^20")
    eip2537_case(16, "eip2537_g1_msm_2^16")
    blob_case("eip4844_blob_4096")
    return out


def _tau(seed: int) -> bytes:
    import crypto_b200 as kb
    return kb.gen_scalars(CURVE, seed, 1)


def bench_batched_commits(args) -> dict:
    """512 BLS12-381 commits, sizes log-uniform over 2^8..2^16 (powers of
    two), uniform Fr evaluations, one resident 2^16 SRS: the batched pass
    (grouped iNTTs + one batched MSM, CUDA graph) against 512 sequential
    plain kzg_commit_fr calls on the same GPU, byte-equal.  The autotuner
    first times the candidate commit windows, MSM windows and NTT radix
    splits of every size class on this GPU (kb200_autotune), writes its
    cache, and the run loads it (kb200_autotune_load): both forms then use
    the tuned choices, reported under "autotune"."""
    import random
    import crypto_b200 as kb
    L = kb.lib()
    rng = random.Random(4096)
    sizes = [1 << rng.randint(8, 16) for _ in range(args.commits)]
    kb.kzg_srs_generate(_tau(7), 1 << 16)
    fd, cache = tempfile.mkstemp(suffix=".tune")
    os.close(fd)
    t0 = time.perf_counter()
    tuned = L.kb200_autotune(CURVE, 8, 16, cache.encode())
    tune_s = time.perf_counter() - t0
    for kind in range(4):  # start from empty tables, then apply the cache
        for lg in range(8, 17):
            L.kb200_tune_set(kind, CURVE, lg, 0)
    applied = L.kb200_autotune_load(cache.encode())
    os.unlink(cache)
    choices = {str(lg): {"commit_window": L.kb200_tune_get(3, CURVE, lg),
                         "msm_window": L.kb200_tune_get(0, CURVE, lg),
                         "msm_glv_window": L.kb200_tune_get(2, CURVE, lg),
                         "ntt_first_pass_log_radix": L.kb200_tune_get(1, CURVE, lg)}
               for lg in range(8, 17)}
    # new commit windows may need their shifted tables and larger engines:
    # the setup builds and warms them before anything is timed
    kb.kzg_srs_generate(_tau(7), 1 << 16)
    evs = [kb.gen_scalars(CURVE, 100000 + i, n) for i, n in enumerate(sizes)]
    blob = b"".join(evs)
    # per-call: every commit through the plain C ABI, host buffers
    kb.kzg_commit(evs[0])
    t0 = time.perf_counter()
    single = [kb.kzg_commit(e) for e in evs]
    t_single = time.perf_counter() - t0
    # batched: one call per 512-commit batch (graph captured on the first)
    batch = kb.kzg_commit_batch(blob, sizes)
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        batch = kb.kzg_commit_batch(blob, sizes)
    t_batch = (time.perf_counter() - t0) / reps
    return {"commits": len(sizes), "sizes": "2^8..2^16 log-uniform", "srs": "2^16 resident",
            "autotune": {"size_classes": tuned, "entries_applied": applied, "seconds": tune_s,
                         "choices_by_log_n": choices},
            "per_call_commits_per_s": len(sizes) / t_single,
            "batched_commits_per_s": len(sizes) / t_batch,
            "batched_over_per_call": t_single / t_batch,
            "byte_equal": batch == single, "h2d_bytes": len(blob), "d2h_bytes": 48 * len(sizes)}


def bench_served_commits(args) -> dict:
    """Poisson arrivals of commit requests (70% 4096, 25% 2^16, 5% 2^20
    evaluations) against a resident 2^20 SRS through the continuous-batching
    server; p50/p99 submit-to-result latency and sustained commits/s per
    arrival rate, results byte-checked against the plain path."""
    import random
    import threading
    import crypto_b200 as kb
    kb.kzg_srs_generate(_tau(8), 1 << 20)
    pool = {}
    for n in (4096, 1 << 16, 1 << 20):
        pool[n] = [kb.gen_scalars(CURVE, 200000 + n + j, n) for j in range(3)]
    want = {(n, j): kb.kzg_commit(e) for n, es in pool.items() for j, e in enumerate(es)}
    out = []
    for rate in args.serve_rates:
        rng = random.Random(int(rate))
        reqs = []
        for _ in range(args.serve_requests):
            u = rng.random()
            n = 4096 if u < 0.70 else ((1 << 16) if u < 0.95 else (1 << 20))
            reqs.append((n, rng.randrange(3), rng.expovariate(rate)))
        ok = True
        with kb.KzgServer(max_batch=64, slots=2) as srv:
            tickets = []

            def producer():
                t_next = time.perf_counter()
                for n, j, gap in reqs:
                    t_next += gap
                    d = t_next - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    tickets.append(((n, j), srv.submit(pool[n][j])))

            th = threading.Thread(target=producer)
            t0 = time.perf_counter()
            th.start()
            th.join()
            for key, t in tickets:
                c, _ms = srv.wait(t, timeout_ms=120000)
                ok &= (c == want[key])
            wall = time.perf_counter() - t0
            st = srv.stats()
        out.append({"rate_per_s": rate, "requests": len(reqs), "p50_ms": st["p50_ms"],
                    "p99_ms": st["p99_ms"], "commits_per_s": st["commits_per_s"],
                    "wall_s": wall, "byte_equal": ok})
    # the knee: the highest offered rate the server still sustains (>= 95% of
    # it completed per second); above it the queue grows and latency with it
    kept = [r for r in out if r["commits_per_s"] >= 0.95 * r["rate_per_s"]]
    knee = max(kept, key=lambda r: r["rate_per_s"]) if kept else None
    return {"mix": "70% 4096 / 25% 2^16 / 5% 2^20", "srs": "2^20 resident", "rates": out,
            "knee_rate_per_s": knee["rate_per_s"] if knee else None,
            "knee_p99_ms": knee["p99_ms"] if knee else None,
            "saturation_commits_per_s": max(r["commits_per_s"] for r in out) if out else None}


def run_reference(args, ws, rank):
    """The reference arm: the reference's own CPU MSM on the headline
    workload, built and run on the host (rank 0 only; other ranks exit
    without work).  Never loads the CUDA library."""
    if rank != 0:
        return
    import _oracle as O
    n = 1 << args.logn
    threads = ref_threads()
    scs, pts = cpu_workload(n)
    nblocks = max(1, n >> REF_BLOCK_LOG)
    for i in range(args.warmup):
        ref_block(scs, pts, n, i, threads)
    times, sums = [], {}
    for i in range(args.steps):
        dt, r = ref_block(scs, pts, n, args.warmup + i, threads)
        times.append(dt)
        sums[(args.warmup + i) % nblocks] = r
    t = sum(times) / len(times)
    m = min(n, 1 << REF_BLOCK_LOG)
    v = m / t / 1e6
    check = None
    want = golden_expected(args.logn)
    if want and len(sums) == nblocks:
        acc = bytes(PB)
        for b in range(nblocks):
            acc = O.g1_add(CURVE, acc, sums[b])
        check = acc.hex() == want
    line = {
        "impl": "reference", "metric": "G1 MSM Mpts/s @2^22", "value": v, "unit": "Mpts/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": headline_config(args.logn),
        "cpu_baseline": {"value": v, "unit": "Mpts/s", "cores": threads, "kind": "reference",
                         "sample": ref_sample_text(n, threads)},
        "e2e": {"value": v, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "block_sums_match_golden": check,
    }
    print(json.dumps(line), flush=True)


def cpu_baselines(args, host_sc: bytes, host_pts: bytes) -> dict:
    """The CPU baselines of the other configurations, timed on this host:
    the reference MSM as shipped (one thread), the restated Fr NTT (the
    reference has none), the plain KZG commit (restated iNTT -> the reference
    MSM -> restated encoder), and the batched and served commit mixes spread
    over all host cores.  Each is a bounded sample, said in its entry."""
    import random
    import concurrent.futures as cf
    import _oracle as O
    cores = ref_threads()
    out = {}
    # the reference MSM as shipped runs on one thread: the first 2^16 points
    # of the headline workload (~4 s), at the window it picks for 2^16 points
    m = min(len(host_sc) // 32, 1 << 16)
    t0 = time.perf_counter()
    O.ref_msm(CURVE, host_sc[:32 * m], host_pts[:PB * m], m)
    t = time.perf_counter() - t0
    out["msm_reference_1_core"] = {
        "mpts_per_s": m / t / 1e6, "cores": 1, "kind": "reference",
        "sample": f"gpukit_multi_pippenger_cpu (built unmodified from its sources) on the first {m} "
                  f"points of the headline workload, one thread, as the reference ships it"}
    # Fr NTT forward, BLS12-381 (restated radix-2, one core): a 2^22 sample
    # of the 2^24 configuration (one 2^24 transform takes ~40 s on one core)
    n = 1 << 22
    x = O.gen_scalars(CURVE, 5 + 22, n)
    buf = ctypes.create_string_buffer(x, len(x))
    t0 = time.perf_counter()
    assert O.orc().orc_ntt(CURVE, buf, n, 0, 0) == 0
    t = time.perf_counter() - t0
    out["fr_ntt_bls12_381_2^22"] = {
        "ms_forward": t * 1e3, "butterflies_per_s": (n // 2) * 22 / t, "cores": 1, "kind": "port",
        "sample": "one 2^22 forward transform (oracle orc_ntt, radix-2 restatement; the reference "
                  "has no Fr NTT) standing in for the 2^24 configuration"}
    del buf, x

    # KZG commit kernels shared by the commit baselines: SRS [tau^i]G1
    tau = bytes(O.gen_scalars(CURVE, 7, 1))
    srs = O.fixed_base_points(CURVE, O.fr_powers(CURVE, tau, 1 << 16))

    def commit(ev: bytes) -> bytes:
        m = len(ev) // 32
        coeffs = O.ntt(CURVE, ev, inverse=True)
        return O.compress(O.ref_msm(CURVE, coeffs, srs[:96 * m], m))

    ev = O.gen_scalars(CURVE, 4096, 4096)
    commit(ev)
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        commit(ev)
    t = (time.perf_counter() - t0) / reps
    out["kzg_commit_4096"] = {"ms": t * 1e3, "commits_per_s": 1 / t, "cores": 1, "kind": "reference",
                              "sample": "restated iNTT -> reference gpukit_multi_pippenger_cpu -> restated "
                                        "compressed encoder, one commit of 4096 evaluations, 3 repetitions"}

    # 512 uneven commits (2^8..2^16): every 8th commit of the benchmark's size
    # list, spread over all cores (ctypes calls release the GIL)
    rng = random.Random(4096)
    sizes = [1 << rng.randint(8, 16) for _ in range(args.commits)][::8]
    evs = [O.gen_scalars(CURVE, 100000 + 8 * i, m) for i, m in enumerate(sizes)]
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(cores) as ex:
        list(ex.map(commit, evs))
    t = time.perf_counter() - t0
    out["kzg_batched_uneven"] = {"commits_per_s": len(sizes) / t, "cores": cores, "kind": "reference",
                                 "sample": f"{len(sizes)} of the 512 commits (every 8th of the same size "
                                           f"list), one commit per core at a time"}

    # served mix (70% 4096, 25% 2^16, 5% 2^20): service time per class
    lat = {}
    for m in (4096, 1 << 16):
        e = O.gen_scalars(CURVE, 200000 + m, m)
        t0 = time.perf_counter()
        commit(e)
        lat[m] = time.perf_counter() - t0
    m = 1 << 20
    big_srs = O.fixed_base_points(CURVE, O.fr_powers(CURVE, tau, m))
    e = O.gen_scalars(CURVE, 200000 + m, m)
    t0 = time.perf_counter()
    coeffs = O.ntt(CURVE, e, inverse=True)
    O.compress(O.ref_msm(CURVE, coeffs, big_srs, m, threads=cores))
    t_big = time.perf_counter() - t0
    mean_1core = 0.70 * lat[4096] + 0.25 * lat[1 << 16] + 0.05 * t_big * cores
    out["kzg_served_mix"] = {
        "service_ms": {"4096 (1 core)": lat[4096] * 1e3, "65536 (1 core)": lat[1 << 16] * 1e3,
                       f"1048576 ({cores} cores)": t_big * 1e3},
        "commits_per_s_all_cores": cores / mean_1core, "cores": cores, "kind": "reference",
        "sample": "one commit per size class; the mix's throughput on all cores is derived as "
                  "cores / mean single-core service time, the 2^20 class counted as its all-core "
                  "time x cores"}
    return out


def run_ours(args, ws, rank, local):
    import torch
    import crypto_b200 as kb
    n = 1 << args.logn
    d_sc, d_pts = make_inputs(n, seed=SCALAR_SEED + rank)
    d_out = torch.empty(PB, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    L = kb.lib()
    # The drop-in path (exact for every curve point: 256-bit windows on
    # BLS12-381) and the G1-promise path (GLV split), both on device buffers.
    dev_fn = {"plain": L.kb200_msm_device, "subgroup": L.kb200_msm_device_subgroup}
    host_fn = {"plain": L.gpukit_multi_pippenger, "subgroup": L.gpukit_multi_pippenger_subgroup}
    head = args.path
    other = "subgroup" if head == "plain" else "plain"

    def run(path):
        rc = dev_fn[path](CURVE, d_sc.data_ptr(), d_pts.data_ptr(), n, d_out.data_ptr(), sp)
        assert rc == 0, kb.last_error()

    # warm-up of both paths; their sums against the reference's (the golden
    # sum of the same workload from the reference CPU MSM) and each other
    want = golden_expected(args.logn) if rank == 0 else None
    sums = {}
    for path in ((head,) if args.single_path else (other, head)):
        for _ in range(args.warmup):
            run(path)
        torch.cuda.synchronize()
        sums[path] = d_out.cpu().numpy().tobytes()
    if not args.single_path:
        assert sums["plain"] == sums["subgroup"], "the two MSM paths disagree"
    parity = {"reference_sum_equal": (sums[head].hex() == want) if want else None,
              "against": "reference CPU MSM of this workload (tests/golden/large.json)"}
    if want:
        assert sums[head].hex() == want, "MSM differs from the reference's sum"
    host_sc = d_sc.cpu().numpy().tobytes()
    host_pts = d_pts.cpu().numpy().tobytes()

    def timed(path, steps, sample_clocks):
        kb.profile_enable(True)
        barrier(ws)
        torch.cuda.synchronize()
        launches0 = kb.launch_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        clk = ClockSampler(torch.cuda.current_device()) if sample_clocks else None
        if clk:
            clk.__enter__()
        try:
            ev0.record(stream)
            for _ in range(steps):
                run(path)
            ev1.record(stream)
            torch.cuda.synchronize()
        finally:
            if clk:
                clk.__exit__()
        launches = kb.launch_count() - launches0
        barrier(ws)
        stage = kb.msm_stage_ms(CURVE)
        kb.profile_enable(False)
        ms = max_over_ranks(ws, ev0.elapsed_time(ev1) / steps)
        return ms, launches, stage, (clk.summary() if clk else None)

    ms, launches, stage, clocks = timed(head, args.steps, True)
    value = n * ws / (ms / 1e3) / 1e6

    # e2e through the C ABI with pinned host buffers (copies in the timed region)
    h_sc = torch.frombuffer(bytearray(host_sc), dtype=torch.uint8).pin_memory()
    h_pts = torch.frombuffer(bytearray(host_pts), dtype=torch.uint8).pin_memory()
    out = ctypes.create_string_buffer(PB)

    def e2e(path):
        f = host_fn[path]
        steps = max(1, min(args.steps, 5))
        assert f(CURVE, ctypes.c_char_p(h_sc.data_ptr()), ctypes.c_char_p(h_pts.data_ptr()), n, out) == 0
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(steps):
            rc = f(CURVE, ctypes.c_char_p(h_sc.data_ptr()), ctypes.c_char_p(h_pts.data_ptr()), n, out)
            assert rc == 0, kb.last_error()
        e_ms = max_over_ranks(ws, (time.perf_counter() - t0) * 1e3 / steps)
        assert out.raw == sums[path]
        return e_ms

    e2e_ms = e2e(head)

    peaks = load_peaks()
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    peak_imad = SM_COUNT * IMAD_PER_CLK_SM * sm_mhz * 1e6

    def rooflines(path, stage_ms, step_ms):
        # dominant phase: the bucket accumulation, i.e. the batch-affine pairing
        # levels (k_pair_fwd, k_inv_wide, k_pair_bwd) and the XYZZ accumulation of
        # what they leave (k_accumulate), timed by the stage events around both
        entries = (L.kb200_msm_entries_subgroup if path == "subgroup" else L.kb200_msm_entries)(CURVE, n)
        acc_ms = (stage_ms.get("pair") or 0.0) + (stage_ms.get("accumulate") or 0.0)
        roof = None
        if acc_ms > 0:
            ach = entries * 6 * mont_imad(N_LIMBS) / (acc_ms / 1e3)
            roof = {"bound": "int",
                    "kernel": "bucket accumulation: pairing levels (k_pair_fwd, k_inv_wide, k_pair_bwd) "
                              "+ k_accumulate",
                    "achieved": ach / 1e12, "peak": peak_imad / 1e12, "unit": "TIMAD/s",
                    "frac": ach / peak_imad, "traffic": bucket_traffic(path, entries),
                    "peak_source": f"derived: {SM_COUNT} SMs x {IMAD_PER_CLK_SM} IMAD/clk x "
                                   f"{sm_mhz:.0f} MHz (MEASURED_PEAKS sm_max_mhz, else the B200 maximum)",
                    "work_per_launch": f"{entries:.3e} bucket additions x 6 x {mont_imad(N_LIMBS)} IMAD"}
        msm_w = w_msm(n, N_LIMBS)
        whole = {"achieved": msm_w / (step_ms / 1e3) / 1e12, "peak": peak_imad / 1e12, "unit": "TIMAD/s",
                 "frac": msm_w / (step_ms / 1e3) / peak_imad,
                 "work": f"W_msm(2^{args.logn}) = {msm_w:.3e} IMAD"}
        return roof, whole

    roofline, msm_roof = rooflines(head, stage, ms)
    other_line = None
    if not args.single_path:
        # the other path, same protocol (device time, then e2e)
        o_ms, _, o_stage, _ = timed(other, args.steps, False)
        o_e2e = e2e(other)
        o_roof, o_whole = rooflines(other, o_stage, o_ms)
        other_line = {"path": other, "value": n * ws / (o_ms / 1e3) / 1e6, "unit": "Mpts/s",
                      "ms_per_step": o_ms, "window_bits": kb.msm_window(CURVE, n, subgroup=(other == "subgroup")),
                      "e2e": {"value": n * ws / (o_e2e / 1e3) / 1e6, "unit": "Mpts/s", "ms_per_step": o_e2e,
                              "api": host_fn[other].__name__},
                      "roofline_frac": o_roof["frac"] if o_roof else None,
                      "msm_roofline_frac": o_whole["frac"], "stage_ms": o_stage}

    extra = None
    if rank == 0 and not args.no_extra:
        extra = bench_extra(args, peak_imad)

    kzg_batched = kzg_served = None
    if rank == 0 and not args.no_kzg:
        kzg_batched = bench_batched_commits(args)
        kzg_served = bench_served_commits(args)

    cpu = cpu_more = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = ref_threads()
        t, _ = ref_block(host_sc, host_pts, n, 0, threads)
        m = min(n, 1 << REF_BLOCK_LOG)
        cpu = {"value": m / t / 1e6, "unit": "Mpts/s", "cores": threads, "kind": "reference",
               "sample": "one step of the reference arm: " + ref_sample_text(n, threads)}
        cpu_more = cpu_baselines(args, host_sc, host_pts)

    if rank == 0:
        line = {
            "metric": "G1 MSM Mpts/s @2^22", "value": value, "unit": "Mpts/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": headline_config(args.logn),
            "path": {"plain": "kb200_msm_device / gpukit_multi_pippenger: exact for every curve point "
                              "(256-bit signed windows on BLS12-381)",
                     "subgroup": "kb200_msm_device_subgroup / gpukit_multi_pippenger_subgroup: points "
                                 "promised in G1 (GLV split)"}[head],
            "window_bits": kb.msm_window(CURVE, n, subgroup=(head == "subgroup")),
            "l2": "inputs 512 MiB > L2 (no flush)", "parallelism": f"replicas x{ws}",
            "parity": parity,
            "e2e": {"value": n * ws / (e2e_ms / 1e3) / 1e6, "unit": "Mpts/s",
                    "h2d_bytes_per_step": n * (32 + PB), "d2h_bytes_per_step": PB,
                    "ms_per_step": e2e_ms, "api": host_fn[head].__name__},
            "gpu_launches": launches,
            "roofline": roofline,
            "msm_roofline": msm_roof,
            "stage_ms": stage,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "msm_other_path": other_line,
            "configs": extra,
            "kzg_batched": kzg_batched,
            "kzg_served": kzg_served,
            "cpu_baselines": cpu_more,
        }
        print(json.dumps(line), flush=True)


def bucket_traffic(path, entries):
    """DRAM bytes of one MSM's bucket accumulation (every pairing-level and
    accumulation launch): dram__bytes_read.sum + dram__bytes_write.sum summed
    over those launches of one smaller MSM of the same path in an ncu
    capture (profiles/msm_bucket_phase_dram.json), scaled by the number of
    sorted entries (the phase's traffic grows with them)."""
    p = ROOT / "profiles" / "msm_bucket_phase_dram.json"
    if CURVE != 2 or not p.exists():
        return None
    d = json.loads(p.read_text()).get(f"bls12_381_{path}")
    if not d:
        return None
    return (d["dram_read"] + d["dram_write"]) * entries / d["entries"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--logn", type=int, default=LOGN)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-kzg", action="store_true")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--case", default="msm", choices=["msm", "ntt"],
                    help="msm: the benchmark line; ntt: one Fr NTT size only (profiling)")
    ap.add_argument("--path", default="plain", choices=["plain", "subgroup"],
                    help="headline MSM entry point: plain (exact for every point) or subgroup (GLV)")
    ap.add_argument("--ntt-curve", type=int, default=CURVE, choices=[1, 2], help="--case ntt: curve")
    ap.add_argument("--coset", action="store_true", help="--case ntt: coset transform")
    ap.add_argument("--single-path", action="store_true",
                    help="time only the --path entry point (profiling runs)")
    ap.add_argument("--commits", type=int, default=512)
    ap.add_argument("--serve-rates", type=float, nargs="*",
                    default=[100.0, 200.0, 400.0, 800.0, 1200.0, 1600.0, 2400.0])
    ap.add_argument("--serve-requests", type=int, default=1000)
    args = ap.parse_args()
    sys.path.insert(0, str(ROOT / "tests"))
    if args.impl == "reference":
        # host-only: no process group, no CUDA context, no CUDA library
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = setup_dist()
    try:
        if args.case == "ntt":
            # a single Fr NTT size, forward + inverse (for profiling the pass kernel)
            import torch
            import crypto_b200 as kb
            n = 1 << args.logn
            curve = args.ntt_curve
            x = kb.gen_scalars(curve, 5, n)
            d = torch.frombuffer(bytearray(x), dtype=torch.uint8).cuda()
            sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            co = int(args.coset)

            def fwd_inv():
                assert kb.lib().kb200_ntt_device(curve, d.data_ptr(), n, 0, co, 1, sp) == 0
                assert kb.lib().kb200_ntt_device(curve, d.data_ptr(), n, 1, co, 1, sp) == 0

            ms = time_device(fwd_inv, args.steps, args.warmup)
            assert d.cpu().numpy().tobytes() == x
            print(json.dumps({"case": "ntt", "curve": {1: "BN254", 2: "BLS12-381"}[curve], "n": n,
                              "coset": bool(co), "ms_fwd_plus_inv": ms,
                              "imad_frac": 2 * w_ntt(n) / (ms / 1e3) / (SM_COUNT * IMAD_PER_CLK_SM * 1965e6)}))
            return
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
