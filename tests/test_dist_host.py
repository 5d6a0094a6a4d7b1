"""Multi-process host logic of bench.py on CPU (gloo, world size 2): the replica timing is the
maximum over ranks, the barrier completes, and the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    dist, r, w = bench._dist()
    assert (r, w) == (rank, ws)
    bench._barrier(dist)
    m = bench._max_over_ranks(dist, 1.5 + rank)
    # the reference arm returns at once on ranks other than 0 (rank 0 would time the oracle)
    ran = None
    if rank != 0:
        bench.run_reference(None, dist, rank, ws)
        ran = False
    bench._barrier(dist)
    dist.destroy_process_group()
    out.put((rank, m, ran))


def test_max_over_ranks_and_barrier_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [m for _, m, _ in res] == [2.5, 2.5]
    assert res[1][2] is False
