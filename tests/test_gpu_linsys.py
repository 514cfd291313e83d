"""A system read from a Linear System Save file set (tests/golden/linsys_hex4_*.dat, laid out as
ElmerSolver's SaveLinearSystem writes it, SolverUtils.src:8588-8662) is bound and solved on the
device and checked against the oracle on the same loaded arrays: SpMV within 1e-14 of the row's
|a||x| scale, ILU0 factors bit-exact, BiCGStab + ILU0 solutions (FP64 and mixed) within 1e-8 and
the FP64 iteration count within one."""
import os

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import linsys_io
from helpers import rel

pytestmark = pytest.mark.gpu
PREFIX = os.path.join(os.path.dirname(__file__), "golden", "linsys_hex4")


def test_saved_system_solves_like_the_oracle(ctx):
    q, v, b = linsys_io.load_linear_system(PREFIX)
    op = oracle.Pattern(q.n, q.nnz, 1, q.perm, q.rows, q.cols, q.diag, 0, 0, 0, 0)
    A = eg.Matrix(ctx, q, v)
    try:
        u = np.random.default_rng(7).standard_normal(q.n)
        scale = oracle.spmv(op, np.abs(v), np.abs(u))
        assert np.max(np.abs(A.mv(u) - oracle.spmv(op, v, u)) / scale) < 1e-14
        ilu, _ = A.ilu0(scale_system=True)
        vs = v.copy()
        oracle.scale(op, vs)
        assert np.array_equal(ilu, oracle.ilu0(op, vs))
        x_ref, r_ref = oracle.solve(op, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, max_iter=500,
                                    tol=1e-10)
        assert r_ref["info"] == 1
        for precision in (eg.FP64, eg.MIXED):
            x, r = A.solve(b, params=eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=500,
                                                     tol=1e-10, precision=precision))
            assert r["info"] == 1
            if precision == eg.FP64:
                assert abs(r["iters"] - r_ref["iters"]) <= 1
            assert rel(x, x_ref) < 1e-8
    finally:
        A.free()
