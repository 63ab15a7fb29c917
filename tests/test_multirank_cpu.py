"""bench.py's multi-rank plumbing on the CPU: two ranks over gloo (the GPU run
uses NCCL, one rank per GPU, through the same helpers). Each rank times its
own replica; the reported time is the slowest rank's, so max_over_ranks must
return the maximum on every rank, and barrier must return on both."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r, w, _ = bench.init_dist(None, backend="gloo")
    bench.barrier(w)
    slowest = bench.max_over_ranks(10.0 + r, w)        # rank r "took" 10 + r ms
    single = bench.max_over_ranks(3.0, 1)             # one rank: the value itself
    bench.barrier(w)
    bench._PG.destroy_process_group()
    out.put((r, w, slowest, single))


def test_two_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    got = sorted(out.get(timeout=10) for _ in range(2))
    assert [g[0] for g in got] == [0, 1]
    for r, w, slowest, single in got:
        assert w == 2 and slowest == 11.0 and single == 3.0
