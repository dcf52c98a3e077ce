"""The multi-rank path of bench.py on CPU: two gloo ranks (one process each, as torchrun starts
them) agree on the maximum of their step times, pass barriers together and take disjoint slices
of the seeded workload. The GPU path is the same code over NCCL."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), MONTMUL_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init(timeout_s=60)
    assert (w, r) == (world, rank)
    bench.barrier(w)
    t = bench.allmax(1.5 + rank, w)
    lo, hi = bench.shard(10, w, r)
    bench.barrier(w)
    out.put((rank, t, lo, hi, dist.get_backend()))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2.5, 0, 10, "gloo"), (1, 2.5, 10, 20, "gloo")]


def test_single_rank_needs_no_process_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_init()[0] == 1
    assert bench.allmax(3.0, 1) == 3.0
    assert bench.shard(7, 1, 0) == (0, 7)
