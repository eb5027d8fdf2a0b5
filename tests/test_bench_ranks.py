"""bench.py's multi-process plumbing on CPU: two gloo ranks, as torchrun launches the
replicas (one process per GPU), agree on the barrier and on the max-over-ranks timing,
and only rank 0 runs the reference arm."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench._barrier(dist)
        worst = bench._max_over_ranks(dist, 10.0 + rank)  # each rank's own time
        skipped = bench.run_reference(None, rank) if rank != 0 else None
        out.put((rank, worst, skipped))
        bench._barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_rank0_alone_reports():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]  # max over ranks, on every rank
    assert res[1][2] is None  # rank 1: no reference work, nothing to print
