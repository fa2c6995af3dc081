"""The multi-GPU path of bench.py is replicas only: every rank solves its own
copy of the system, the reported time is the maximum over ranks, and under
the reference arm only rank 0 works.  This runs that plumbing (process group
set-up by bench.dist_init, max over ranks, barrier, rank-0-only reference)
as two gloo ranks on the CPU."""

import argparse
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "draugr.jl_b200"))
    import torch.distributed as dist

    import bench

    args = argparse.Namespace(impl="reference", n=8, seed=1, steps=1, warmup=0)
    w, r, _ = bench.dist_init(args)  # the reference arm uses gloo
    try:
        backend = dist.get_backend()
        m = bench.max_over_ranks(float(10 * (r + 1)), w)
        bench.barrier(w)
        out = bench.run_reference(args, w, r) if r != 0 else "rank 0 runs the reference"
        q.put((r, w, backend, m, out))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[0] for g in got] == [0, 1]
    for r, w, backend, m, out in got:
        assert w == 2 and backend == "gloo"
        assert m == 20.0  # the max over ranks reaches every rank
    assert got[1][4] is None  # rank 1 of the reference arm does no work
