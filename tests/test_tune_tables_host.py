"""CPU-side checks of the per-size tuning tables the autotuner fills
(crypto_b200/csrc/autotune.cu, msm.cu): an entry set for one (curve, log2 n)
replaces the cost model's MSM window for exactly that size class, 0 gives the
choice back to the cost model, the table consulted is the one of the path the
call takes (GLV halves or 256-bit windows), and out-of-range keys are ignored.  The
planner and the tables are host code, so none of this needs a GPU."""
from __future__ import annotations

import pytest


def kb():
    import crypto_b200
    return crypto_b200


MSM, NTT, MSM_GLV, COMMIT = 0, 1, 2, 3


@pytest.mark.parametrize("curve", [1, 2])
@pytest.mark.parametrize("subgroup", [False, True])
def test_msm_entry_overrides_one_size_class(curve, subgroup):
    L = kb().lib()
    # the wire path splits by GLV on BN254 always (every curve point is in
    # G1 there) and on BLS12-381 when the caller promises G1
    kind = MSM_GLV if subgroup or curve == 1 else MSM
    n = 1 << 18
    model = kb().msm_window(curve, n, subgroup=subgroup)
    below = kb().msm_window(curve, n >> 1, subgroup=subgroup)
    forced = 9 if model != 9 else 10
    try:
        L.kb200_tune_set(kind, curve, 18, forced)
        assert L.kb200_tune_get(kind, curve, 18) == forced
        # sizes 2^17 + 1 .. 2^18 round up to the class 18
        assert kb().msm_window(curve, n, subgroup=subgroup) == forced
        assert kb().msm_window(curve, (n >> 1) + 1, subgroup=subgroup) == forced
        assert kb().msm_window(curve, n >> 1, subgroup=subgroup) == below
        # the other path's table is untouched
        other = MSM if kind == MSM_GLV else MSM_GLV
        assert L.kb200_tune_get(other, curve, 18) == 0
    finally:
        L.kb200_tune_set(kind, curve, 18, 0)
    assert L.kb200_tune_get(kind, curve, 18) == 0
    assert kb().msm_window(curve, n, subgroup=subgroup) == model


def test_out_of_range_keys_ignored():
    L = kb().lib()
    for kind in (MSM, NTT, MSM_GLV):
        for curve, lg in ((0, 10), (3, 10), (1, -1), (1, 48)):
            L.kb200_tune_set(kind, curve, lg, 7)
            assert L.kb200_tune_get(kind, curve, lg) == 0
    # commit windows exist for BLS12-381 (curve 2) only
    L.kb200_tune_set(COMMIT, 1, 12, 16)
    assert L.kb200_tune_get(COMMIT, 1, 12) == 0
    # and only at the widths the shifted tables are built for (13, 16, 19)
    L.kb200_tune_set(COMMIT, 2, 12, 14)
    assert L.kb200_tune_get(COMMIT, 2, 12) == 0
    assert L.kb200_tune_get(99, 2, 12) == 0


def test_ntt_and_commit_entries_round_trip():
    L = kb().lib()
    try:
        L.kb200_tune_set(NTT, 2, 20, 8)
        L.kb200_tune_set(COMMIT, 2, 12, 16)
        assert L.kb200_tune_get(NTT, 2, 20) == 8
        assert L.kb200_tune_get(NTT, 1, 20) == 0
        assert L.kb200_tune_get(COMMIT, 2, 12) == 16
    finally:
        L.kb200_tune_set(NTT, 2, 20, 0)
        L.kb200_tune_set(COMMIT, 2, 12, 0)
    assert L.kb200_tune_get(NTT, 2, 20) == 0
    assert L.kb200_tune_get(COMMIT, 2, 12) == 0
