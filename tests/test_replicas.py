"""Multi-GPU runs are replicas (independent systems per rank, no data-path collective):
the bench's rendezvous, barrier and max-over-ranks timing on 2 gloo ranks (CPU)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), BENCH_BACKEND="gloo")
    import bench

    r, w, local, pg = bench.dist_setup(world)
    assert (r, w, local) == (rank, world, rank)
    bench.barrier(pg, None)
    t = bench.reduce_max(pg, 1.0 + rank, None)
    out.put((rank, t))
    pg.destroy_process_group()


def test_two_rank_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 2.0, 1: 2.0}
