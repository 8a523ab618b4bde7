"""bench.py --gpus N runs N replicas, one rank per GPU: the rank plumbing
(process group, barrier around the timed region, max-over-ranks timing, the
reference arm on rank 0 only) as world_size-2 gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, ws: int, port: int, q) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench
    try:
        w, r, _ = bench.setup_dist()
        bench.barrier(w)
        # each rank's step time; the aggregate uses the slowest rank
        slowest = bench.max_over_ranks(w, 10.0 + 5.0 * r)
        bench.barrier(w)
        q.put((r, w, dist.get_backend(), slowest))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_two_rank_barrier_and_max_over_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert got == [(0, 2, "gloo", 15.0), (1, 2, "gloo", 15.0)]
    assert all(p.exitcode == 0 for p in procs)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun the reference arm's other ranks exit without work or output."""
    sys.path.insert(0, str(ROOT))
    import argparse

    import bench
    args = argparse.Namespace(logn=10, steps=1, warmup=0, gpus=2)
    assert bench.run_reference(args, 2, 1) is None
    assert capsys.readouterr().out == ""
