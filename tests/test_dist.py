"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the barrier
and the max over ranks that turn per-rank device times into the whole-job
number, as torchrun launches it (one process per GPU, 127.0.0.1 rendezvous)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, loc = bench.dist_setup()
    d = bench.Dist(w, loc, backend="gloo")
    d.barrier()
    ms = 10.0 + 5.0 * r          # rank 1 is the slow one
    m = d.max(ms)
    v = bench.aggregate_value(256 ** 3, 100, w, m)
    d.barrier()
    d.close()
    out.put((r, m, v))


def test_two_rank_max_and_value():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for r, m, v in res:
        assert m == 15.0
        assert v == pytest.approx(256 ** 3 * 100 * 2 / 0.015 / 1e9)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(1, 0)
    assert d.max(3.5) == 3.5
    d.barrier()
    d.close()
