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


def _fixture():
    import os
    import sys

    here = os.path.join(os.path.dirname(__file__), "golden")
    sys.path.insert(0, here)
    import make_linsys_fixture

    return os.path.join(here, "linsys_hex4"), make_linsys_fixture


def test_loads_files_in_the_reference_layout():
    """tests/golden/linsys_hex4_*.dat is laid out as ElmerSolver's SaveLinearSystem writes it
    (I0 indices, list-directed reals with three-digit exponents such as 8.6232004998696182E-002,
    list-directed integers in the sizes file, '0.0' for a vanishing rhs entry).  The loader
    rebuilds Rows/Cols/Diag/Perm and reads Values and the RHS to the bit of the system the file
    was written from."""
    prefix, mk = _fixture()
    assert "E-00" in open(prefix + "_a.dat").read()
    q, v, b = linsys_io.load_linear_system(prefix)
    p, v0, b0, _ = mk.system()
    assert (q.n, q.nnz) == (p.n, p.nnz)
    for f in ("rows", "cols", "diag", "perm"):
        assert np.array_equal(getattr(q, f), getattr(p, f)), f
    assert np.array_equal(v, v0) and np.array_equal(b, b0)


def test_list_directed_layout_round_trips():
    _, mk = _fixture()
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.standard_normal(200) * 10.0 ** rng.integers(-30, 30, 200),
                         [0.1, 0.09999999999999999, 1e16, 9.999999999999998e15, -1.0, 1e-300, 123456.789]])
    for x in xs:
        s = mk.list_directed_real(x)
        assert float(s) == x, (x, s)
        if abs(x) < 0.1 or abs(x) >= 1e16:
            assert s.strip()[-5] == "E" and s.strip()[-4] in "+-"
