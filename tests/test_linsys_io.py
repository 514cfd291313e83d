"""Linear System Save files: round trip of the exchange format (CPU)."""
import numpy as np

import oracle
from elmerfem_b200 import linsys_io, meshgen
from helpers import poisson_problem


def test_round_trip(tmp_path):
    m = meshgen.tet_cube(3)
    p, _, _, v, b, _ = poisson_problem(m)
    pat = linsys_io.CRSPattern(p.n, p.nnz, 1, p.perm, p.rows, p.cols, p.diag)
    prefix = str(tmp_path / "linsys")
    linsys_io.save_linear_system(prefix, pat, v, b, perm=p.perm)
    q, v2, b2 = linsys_io.load_linear_system(prefix)
    assert np.array_equal(q.rows, p.rows) and np.array_equal(q.cols, p.cols) and np.array_equal(q.diag, p.diag)
    assert np.array_equal(v2, v) and np.array_equal(b2, b) and np.array_equal(q.perm, p.perm)
    x1, r1 = oracle.solve(p, v, b, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=500)
    qp = oracle.Pattern(q.n, q.nnz, 1, q.perm, q.rows, q.cols, q.diag, 0, 0, 0, 0)
    x2, r2 = oracle.solve(qp, v2, b2, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=500)
    assert r1["iters"] == r2["iters"] and np.array_equal(x1, x2)


def test_zero_rhs_written_as_zero(tmp_path):
    m = meshgen.hex_cube(2)
    p, _, _, v, b, _ = poisson_problem(m)
    b[:] = 0.0
    pat = linsys_io.CRSPattern(p.n, p.nnz, 1, p.perm, p.rows, p.cols, p.diag)
    prefix = str(tmp_path / "s")
    linsys_io.save_linear_system(prefix, pat, v, b)
    assert all(l.split()[1] == "0.0" for l in open(prefix + "_b.dat"))
