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


def test_compare_states_counts_cells_and_l1():
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    rng = np.random.default_rng(1)
    ref = (rng.random((50, 3)), rng.random(50) + 1, rng.random((50, 3)), rng.random(50) + 1)
    same = tuple(a.copy() for a in ref)
    r = bench.compare_states(ref, same)
    assert r["cells_differing"] == 0 and all(v == 0.0 for v in r["l1_rel"].values())
    got = tuple(a.copy() for a in ref)
    got[1][7] *= 1 + 1e-12          # one mass
    got[2][9, 2] = np.nextafter(got[2][9, 2], 2.0)  # one momentum component, one ulp
    got[0][7, 0] = np.nan           # the same cell as the mass change
    ref[0][3, 1] = got[0][3, 1] = np.nan  # NaN in both: equal
    r = bench.compare_states(ref, got)
    assert r["cells_differing"] == 2
    assert r["l1_rel"]["mass"] > 0 and r["l1_rel"]["energy"] == 0.0
