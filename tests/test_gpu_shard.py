"""The row-sharded solve's device backend (elmerfem_b200/shard.py) on one GPU: a world of one rank
over NCCL, the whole system one block, so the rank's SpMV (egpu_mv_dev over owned + halo
columns), its Jacobi / block ILU0 (egpu_ilu0_build, egpu_lu_precondition_dev), the scaling and the
HUTI loops run on the device and must match the oracle's plain solve: iterations within one,
solution within 1e-8.  The multi-rank exchange is covered on CPU ranks (test_shard.py); this run
has one GPU."""
import datetime
import os
import socket

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen, shard
from helpers import poisson_problem, rel

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.fixture(scope="module")
def dist_one():
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    yield dist
    dist.destroy_process_group()


@pytest.mark.parametrize("method,prec", [(eg.CG, eg.PREC_DIAGONAL), (eg.BICGSTAB, eg.PREC_ILU0)])
def test_device_backend_one_rank(ctx, dist_one, method, prec):
    import torch

    m = meshgen.hex_cube(10)
    p, _, _, v, b, _ = poisson_problem(m, elem_k=meshgen.lognormal_conductivity(m.nelem, 1.0, 4), sym=True)
    part = shard.RowPartition(p.n, p.rows, p.cols, 1)
    blk = shard.distributed_block(dist_one, part, 0)
    assert blk.nh == 0
    comm = shard.Comm(dist_one, blk, device=torch.device("cuda", 0))
    be = shard.DeviceBackend(ctx, blk, torch.device("cuda", 0))
    x, res = shard.sharded_solve(comm, be, v[blk.src], b, method=method, precond=prec, tol=1e-10, max_iter=2000)
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=prec, max_iter=2000, tol=1e-10)
    assert res["info"] == r_ref["info"] == 1
    assert abs(res["iters"] - r_ref["iters"]) <= 1
    assert rel(x, x_ref) < 1e-8
