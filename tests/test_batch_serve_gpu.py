"""Batched and served commits: byte-equal to the plain per-call path (and to
the oracle), CUDA-graph replay, continuous batching, admission under a
memory budget, and 'same result alone and in the mix'."""
from __future__ import annotations

import random
import threading

import pytest

import _oracle as O

pytestmark = pytest.mark.gpu


def kb():
    import crypto_b200
    return crypto_b200


@pytest.fixture(scope="module")
def srs16(cuda_lib):
    rng = random.Random(77)
    tau = rng.randrange(O.FR[2])
    kb().kzg_srs_generate(tau.to_bytes(32, "little"), 1 << 16)
    return tau


def uneven_sizes(rng: random.Random, count: int, lo: int = 8, hi: int = 16) -> list[int]:
    return [1 << rng.randint(lo, hi) for _ in range(count)]


def test_batch_uneven_equals_per_call(srs16):
    rng = random.Random(1)
    sizes = uneven_sizes(rng, 48)
    evs = [kb().gen_scalars(2, 1000 + i, s) for i, s in enumerate(sizes)]
    batch = kb().kzg_commit_batch(b"".join(evs), sizes)
    for e, c in zip(evs, batch):
        assert kb().kzg_commit(e) == c
    # replay of the captured graph for the same signature gives the same bytes
    assert kb().kzg_commit_batch(b"".join(evs), sizes) == batch
    # a different polynomial set of the same signature reuses the graph
    evs2 = [kb().gen_scalars(2, 5000 + i, s) for i, s in enumerate(sizes)]
    batch2 = kb().kzg_commit_batch(b"".join(evs2), sizes)
    for e, c in zip(evs2[:6], batch2[:6]):
        assert kb().kzg_commit(e) == c


def test_batch_against_oracle_small(srs16):
    rng = random.Random(2)
    sizes = [1 << rng.randint(0, 9) for _ in range(20)]
    srs = kb().kzg_srs_read(0, max(sizes))
    evs = [kb().gen_scalars(2, 3000 + i, s) for i, s in enumerate(sizes)]
    batch = kb().kzg_commit_batch(b"".join(evs), sizes)
    for e, s, c in zip(evs, sizes, batch):
        assert O.kzg_commit(e, srs[:96 * s]) == c


def test_server_same_alone_and_in_mix(srs16):
    rng = random.Random(3)
    sizes = [4096] * 10 + [1 << 16] * 3 + [256] * 10
    rng.shuffle(sizes)
    evs = [kb().gen_scalars(2, 7000 + i, s) for i, s in enumerate(sizes)]
    alone = [kb().kzg_commit(e) for e in evs]
    with kb().KzgServer(max_batch=8, slots=2) as srv:
        # alone: one at a time
        for e, a in zip(evs[:3], alone[:3]):
            t = srv.submit(e)
            c, ms = srv.wait(t, timeout_ms=60000)
            assert c == a and ms > 0
        # in the mix: everything at once from several threads
        results = {}

        def worker(idx):
            for i in idx:
                t = srv.submit(evs[i])
                results[i] = srv.wait(t, timeout_ms=60000)[0]

        th = [threading.Thread(target=worker, args=(list(range(k, len(evs), 4)),)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert [results[i] for i in range(len(evs))] == alone
        st = srv.stats()
        assert st["completed"] >= len(evs) and st["p99_ms"] >= st["p50_ms"] > 0


def test_server_admission_under_budget(srs16):
    """A tight memory budget forces one request per batch; results unchanged."""
    sizes = [1 << 16, 1 << 16, 4096]
    evs = [kb().gen_scalars(2, 9000 + i, s) for i, s in enumerate(sizes)]
    alone = [kb().kzg_commit(e) for e in evs]
    with kb().KzgServer(max_batch=64, slots=1, mem_budget=1) as srv:
        ts = [srv.submit(e) for e in evs]
        got = [srv.wait(t, timeout_ms=60000)[0] for t in ts]
    assert got == alone


def test_server_rejects_bad_sizes(srs16):
    import ctypes
    with kb().KzgServer() as srv:
        t = ctypes.c_uint64()
        assert kb().lib().kzg_server_submit(srv.h, b"\0" * 96, 3, ctypes.byref(t)) == -2
        assert kb().lib().kzg_server_submit(srv.h, b"\0" * 32, 1 << 17, ctypes.byref(t)) == -2
