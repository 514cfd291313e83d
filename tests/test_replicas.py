"""Multi-GPU runs are replicas (independent systems per rank, no data-path collective):
the bench's rendezvous, barrier and max-over-ranks timing on 2 gloo ranks (CPU), and the
reference arm's launch (rank 0 alone, one JSON line) on the CPU."""
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


def test_reference_arm_under_two_ranks_prints_one_line():
    """`bench.py --impl reference` launched like a 2-GPU run: rank 0 alone times the CPU
    reference (the oracle on every host thread) and prints the one JSON line; the other rank
    exits 0 without work."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, BENCH_BACKEND="gloo")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--workload",
           "poisson32_bicgstab_ilu0", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    import time

    t0 = time.perf_counter()
    out = subprocess.run(cmd, cwd=root, env=env, capture_output=True, text=True, timeout=600)
    wall = time.perf_counter() - t0
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(s) for s in out.stdout.splitlines() if s.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    # every step is one whole oracle solve: ms_per_step is a time a step took, and the steps fit
    # in the run's own wall time
    assert abs(d["value"] * d["ms_per_step"] / 1000.0 - 1.0) < 1e-9
    assert d["steps"] * d["ms_per_step"] / 1000.0 < wall
    # the same config as the GPU arm's line (bench.headline_config)
    import bench

    _, _, cfg = bench.workload_spec("poisson32_bicgstab_ilu0")
    assert d["config"] == bench.headline_config(cfg, 33 ** 3, 97 ** 3, 2)
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_of_the_batched_workload():
    """`--impl reference` on the batched workload: the oracle solves the seeded systems one at a
    time and reports systems per second (a short run on 6 systems)."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--workload", "batch512_tet_cg_jacobi", "--systems", "6",
           "--steps", "1", "--warmup", "0"]
    out = subprocess.run(cmd, cwd=root, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(s) for s in out.stdout.splitlines() if s.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0 and d["config"]["systems"] == 6
    assert d["cpu_baseline"]["kind"] == "port" and "seeded order" in d["cpu_baseline"]["sample"]
