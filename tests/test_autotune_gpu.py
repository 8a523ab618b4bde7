"""The autotuner (kb200_autotune / kb200_autotune_load): tune a small range
of sizes on this GPU, write the cache, clear the tables, reload the cache,
and check that every result computed under the tuned parameters (MSM windows
of both paths, NTT radix splits, commit windows) is byte-equal to the
oracle's, as under the cost models' choices."""
from __future__ import annotations

import ctypes

import pytest

import _oracle as O

pytestmark = pytest.mark.gpu


def kb():
    import crypto_b200
    return crypto_b200


def test_autotune_cache_roundtrip_and_results(cuda_lib, tmp_path):
    k = kb()
    L = k.lib()
    lo, hi = 11, 14
    tau = k.gen_scalars(2, 71, 1)
    k.kzg_srs_generate(tau, 1 << hi)
    srs = k.kzg_srs_read(0, 1 << hi)
    # results under the cost models
    cases = []
    for lg in range(lo, hi + 1):
        n = 1 << lg
        ev = k.gen_scalars(2, 500 + lg, n)
        cases.append((lg, ev, k.kzg_commit(ev), k.ntt_fr(1, ev), k.ntt_fr(2, ev, inverse=True)))
    cache = tmp_path / "tune.txt"
    for curve in (1, 2):
        tuned = L.kb200_autotune(curve, lo, hi, str(cache).encode())
        assert tuned == hi - lo + 1, k.last_error()
    lines = cache.read_text().splitlines()
    kinds = {ln.split()[1] for ln in lines}
    assert {"msm", "msm_glv", "ntt", "commit"} <= kinds, kinds
    # clear every table, reload from the cache
    for kind in range(4):
        for curve in (1, 2):
            for lg in range(lo, hi + 1):
                L.kb200_tune_set(kind, curve, lg, 0)
    applied = L.kb200_autotune_load(str(cache).encode())
    assert applied == len(lines)
    for ln in lines:
        _, kind, curve, lg, v = ln.split()[:5]
        knum = {"msm": 0, "ntt": 1, "msm_glv": 2, "commit": 3}[kind]
        assert L.kb200_tune_get(knum, int(curve), int(lg)) == int(v)
    # results under the tuned parameters
    for lg, ev, commit, fwd_bn, inv_bls in cases:
        n = 1 << lg
        assert k.kzg_commit(ev) == commit == O.kzg_commit(ev, srs[:96 * n]), lg
        assert k.ntt_fr(1, ev) == fwd_bn == O.ntt(1, ev), lg
        assert k.ntt_fr(2, ev, inverse=True) == inv_bls, lg
        assert k.kzg_commit_batch(ev + ev, [n, n]) == [commit, commit]
        for curve in (1, 2):
            pts = O.fixed_base_points(curve, O.gen_scalars(curve, 900 + lg, n))
            scs = k.gen_scalars(curve, 901 + lg, n)
            want = O.ref_msm(curve, scs, pts, n, threads=8) if O.ref_available() else O.msm(curve, scs, pts, n)
            assert k.gpukit_multi_pippenger(curve, scs, pts, n) == want, (curve, lg)
            assert k.gpukit_multi_pippenger_subgroup(curve, scs, pts, n) == want, (curve, lg)
    # a forced entry takes effect and stays exact
    L.kb200_tune_set(0, 2, 12, 7)
    assert k.msm_window(2, 1 << 12) == 7
    pts = O.fixed_base_points(2, O.gen_scalars(2, 77, 4096))
    scs = k.gen_scalars(2, 78, 4096)
    assert k.gpukit_multi_pippenger(2, scs, pts, 4096) == O.msm(2, scs, pts, 4096)
    for kind in range(4):
        for curve in (1, 2):
            for lg in range(lo, hi + 1):
                L.kb200_tune_set(kind, curve, lg, 0)


def test_autotune_rejects_bad_ranges(cuda_lib):
    L = kb().lib()
    assert L.kb200_autotune(3, 8, 10, None) < 0
    assert L.kb200_autotune(2, 12, 10, None) < 0
    assert L.kb200_autotune_load(None) < 0
    assert L.kb200_autotune_load(b"/nonexistent/tune.txt") == 0
