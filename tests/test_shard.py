"""Row-block sharding of one system (elmerfem_b200/shard.py) on CPU ranks (gloo).

The device backend needs a GPU per rank; these tests run the same host logic (partition, halo
exchange, global sums, scaling, HUTI CG / BiCGStab) on world-size-2 and -3 gloo ranks with a
CPU stand-in for the rank's compute defined here (a CSR SpMV over owned + halo columns, Jacobi,
and the block's ILU0 restated from CRS_IncompleteLU), and compare with the oracle's
block-Jacobi restatement of the reference's parallel solve (ParILU0 factors each partition's
InsideMatrix, SParIterPrecond.src:234-301): iterations within one and solutions within 1e-8.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from elmerfem_b200 import shard  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(kind):
    import oracle
    from elmerfem_b200 import meshgen
    from helpers import elastic_problem, poisson_problem

    if kind == "hex":
        m = meshgen.hex_cube(7)
        return poisson_problem(m, elem_k=meshgen.lognormal_conductivity(m.nelem, 1.0, 3), sym=True)
    if kind == "tet":
        return poisson_problem(meshgen.tet_cube(6), sym=False)
    return elastic_problem(meshgen.hex_cube(3))


class CpuBlock:
    """Test stand-in for a rank's compute: the block's rows as a dense-free CSR on the host."""

    def __init__(self, block):
        self.block = block
        self.device = "cpu"

    def set_matrix(self, vals, precond):
        b = self.block
        self.vals = np.asarray(vals)
        self.precond = precond
        self.row_of = np.repeat(np.arange(b.nl), np.diff(b.rows))
        if precond == shard.PREC_ILU0:
            self.ilu = self._ilu0(vals)

    def _ilu0(self, vals):
        """CRS_IncompleteLU(A,0) (CRSMatrix.src:2312-2366) of the block's own columns"""
        b = self.block
        keep = b.cols <= b.nl
        rows, cols, v = [], [], []
        for i in range(b.nl):
            sl = slice(b.rows[i] - 1, b.rows[i + 1] - 1)
            c, a = b.cols[sl] - 1, vals[sl]
            k = keep[sl]
            rows.append((c[k], a[k].copy()))
        for i in range(b.nl):
            ci, si = rows[i]
            pos = {int(c): t for t, c in enumerate(ci)}
            for t, k in enumerate(ci):
                if k >= i:
                    break
                if si[t] == 0.0:
                    continue
                ck, sk = rows[k]
                ukk = sk[list(ck).index(k)]
                if abs(ukk) > shard.AEPS:
                    si[t] = si[t] / ukk
                for u, j in enumerate(ck):
                    if j > k and int(j) in pos:
                        si[pos[int(j)]] = si[pos[int(j)]] - si[t] * sk[u]
        for i in range(b.nl):
            ci, si = rows[i]
            d = list(ci).index(i)
            si[d] = 1.0 / si[d] if abs(si[d]) >= shard.AEPS else 1.0
        return rows

    def mv(self, x_full, y):
        x = x_full.numpy()
        out = np.zeros(self.block.nl)
        np.add.at(out, self.row_of, self.vals * x[self.block.cols - 1])
        y.copy_(torch.from_numpy(out))

    def apply_precond(self, v, u):
        b = self.block
        r = v.numpy().copy()
        if self.precond == shard.PREC_ILU0:
            for i in range(b.nl):  # CRS_LUSolve, CRSMatrix.src:3346-3363
                ci, si = self.ilu[i]
                s = r[i]
                for c, a in zip(ci, si):
                    if c < i:
                        s = s - a * r[c]
                r[i] = s
            for i in range(b.nl - 1, -1, -1):
                ci, si = self.ilu[i]
                s = r[i]
                for c, a in zip(ci, si):
                    if c > i:
                        s = s - a * r[c]
                r[i] = si[list(ci).index(i)] * s
        elif self.precond == shard.PREC_DIAGONAL:
            d = np.where(b.diag > 0, self.vals[np.maximum(b.diag, 1) - 1], 0.0)
            r = np.where(np.abs(d) > shard.AEPS, r / np.where(d == 0, 1.0, d), r)
        u.copy_(torch.from_numpy(r))

    def vectors(self, nfull):
        return lambda n: torch.zeros(n, dtype=torch.float64)

    def free(self):
        pass


def _rank_main(rank, world, port, kind, method, precond, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        p, _, _, v, b, _ = _problem(kind)
        part = shard.RowPartition(p.n, p.rows, p.cols, world)
        blk = shard.distributed_block(dist, part, rank)
        comm = shard.Comm(dist, blk)
        x, res = shard.sharded_solve(comm, CpuBlock(blk), v[blk.src], b[blk.r0:blk.r1], method=method,
                                     precond=precond, tol=1e-10, max_iter=2000)
        xs = [None] * world
        dist.all_gather_object(xs, (blk.r0, x))
        if rank == 0:
            out.put((res, xs, [int(s) for s in part.starts]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,kind,method,precond", [
    (2, "hex", shard.CG, shard.PREC_DIAGONAL),
    (2, "hex", shard.BICGSTAB, shard.PREC_ILU0),
    (3, "tet", shard.BICGSTAB, shard.PREC_ILU0),
    (2, "elastic", shard.BICGSTAB, shard.PREC_ILU0),
])
def test_sharded_solve_matches_block_jacobi_oracle(world, kind, method, precond):
    import oracle

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, kind, method, precond, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res, xs, starts = q.get(timeout=300)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p, _, _, v, b, _ = _problem(kind)
    x = np.zeros(p.n)
    for r0, xl in xs:
        x[r0:r0 + len(xl)] = xl
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=precond, max_iter=2000, tol=1e-10,
                                block_starts=starts)
    assert res["info"] == r_ref["info"] == 1
    assert abs(res["iters"] - r_ref["iters"]) <= 1, (res, r_ref)
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-8


def test_partition_halo_and_send_lists():
    """Every rank's local SpMV, fed the halo values its peers send, equals its rows of the
    global product; the send lists are exactly the peers' halos."""
    import oracle

    p, _, _, v, _, _ = _problem("tet")
    part = shard.RowPartition(p.n, p.rows, p.cols, 3)
    assert list(part.starts)[0] == 0 and part.starts[-1] == p.n
    nnz_per = [p.rows[part.starts[k + 1]] - p.rows[part.starts[k]] for k in range(3)]
    assert max(nnz_per) - min(nnz_per) <= 2 * np.max(np.diff(p.rows))
    u = np.random.default_rng(1).standard_normal(p.n)
    ref = oracle.spmv(p, v, u)
    blocks = [part.local(k) for k in range(3)]
    for k, blk in enumerate(blocks):
        full = np.concatenate([u[blk.r0:blk.r1], np.zeros(blk.nh)])
        for q, pos in blk.recv.items():
            sent = blocks[q].send[k]
            assert np.array_equal(blocks[q].r0 + sent, blk.halo[pos])
            full[blk.nl + pos] = u[blocks[q].r0 + sent]
        y = np.zeros(blk.nl)
        np.add.at(y, np.repeat(np.arange(blk.nl), np.diff(blk.rows)), v[blk.src] * full[blk.cols - 1])
        assert np.allclose(y, ref[blk.r0:blk.r1], rtol=1e-14, atol=1e-14 * np.abs(ref).max())
        assert np.all(blk.cols[blk.diag[blk.diag > 0] - 1] == np.nonzero(blk.diag > 0)[0] + 1)


def test_single_block_equals_the_plain_solve():
    """One block: block-Jacobi ILU0 is ILU0, and the oracle's partitioned path equals its plain one."""
    import oracle

    p, _, _, v, b, _ = _problem("hex")
    x1, r1 = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0)
    x2, r2 = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, block_starts=[0, p.n])
    assert r1["iters"] == r2["iters"] and np.array_equal(x1, x2)
