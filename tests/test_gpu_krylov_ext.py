"""GCR and BiCGStab(l) (Linear System Iterative Method = GCR / BiCGStabl) against the oracle.

IterativeMethods.src:919-1055 (GCR with restart) and :559-834 (BiCGStab(l)), run by the
library as persistent FP64 kernels with any of the preconditioners.  The solution must agree
with the oracle's restatement within 1e-8 and the iteration count within one (dot products are
summed in a different order).
"""
import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen
from helpers import elastic_problem, poisson_problem, rel

pytestmark = pytest.mark.gpu


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


PROBLEMS = {
    "hex8": lambda: poisson_problem(meshgen.hex_cube(8)),
    "tet7": lambda: poisson_problem(meshgen.tet_cube(7)),
    "elastic4": lambda: elastic_problem(meshgen.hex_cube(4)),
    "hex14_lognormal": lambda: poisson_problem(meshgen.hex_cube(14),
                                               elem_k=meshgen.lognormal_conductivity(14 ** 3, 1.0, 5)),
}

PRECS = [(eg.PREC_NONE, 0), (eg.PREC_DIAGONAL, 0), (eg.PREC_ILU0, 0), (eg.PREC_ILU0, 1)]


@pytest.mark.parametrize("prec,order", PRECS, ids=["none", "diag", "ilu0", "ilu1"])
@pytest.mark.parametrize("restart", [0, 10])
@pytest.mark.parametrize("name", list(PROBLEMS))
def test_gcr_matches_oracle(ctx, name, restart, prec, order):
    p, _, _, v, b, _ = PROBLEMS[name]()
    tol = 1e-10
    x_ref, r_ref = oracle.solve(p, v, b, method=oracle.GCR, precond=prec, ilu_order=order, max_iter=3000, tol=tol,
                                restart=restart)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, params=eg.SolverParams(method=eg.GCR, precond=prec, ilu_order=order, max_iter=3000, tol=tol,
                                             restart=restart))
    assert r["info"] == 1
    assert abs(r["iters"] - r_ref["iters"]) <= 1, (r["iters"], r_ref["iters"])
    assert rel(x, x_ref) < 1e-8


@pytest.mark.parametrize("prec,order", PRECS, ids=["none", "diag", "ilu0", "ilu1"])
@pytest.mark.parametrize("degree", [2, 4])
@pytest.mark.parametrize("name", list(PROBLEMS))
def test_bicgstabl_matches_oracle(ctx, name, degree, prec, order):
    p, _, _, v, b, _ = PROBLEMS[name]()
    tol = 1e-10
    x_ref, r_ref = oracle.solve(p, v, b, method=oracle.BICGSTABL, precond=prec, ilu_order=order, max_iter=3000,
                                tol=tol, restart=degree)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, params=eg.SolverParams(method=eg.BICGSTABL, precond=prec, ilu_order=order, max_iter=3000,
                                             tol=tol, restart=degree))
    assert r["info"] == 1
    assert abs(r["iters"] - r_ref["iters"]) <= 1, (r["iters"], r_ref["iters"])
    assert rel(x, x_ref) < 1e-8


@pytest.mark.parametrize("mode", ["block", "syncfree"])
@pytest.mark.parametrize("method", [eg.GCR, eg.BICGSTABL], ids=["gcr", "bicgstabl"])
def test_ext_methods_each_tri_mode(ctx, monkeypatch, mode, method):
    monkeypatch.setenv("EGPU_TRI_MODE", mode)
    p, _, _, v, b, _ = PROBLEMS["hex14_lognormal"]()
    omethod = oracle.GCR if method == eg.GCR else oracle.BICGSTABL
    x_ref, r_ref = oracle.solve(p, v, b, method=omethod, precond=eg.PREC_ILU0, max_iter=3000, tol=1e-10)
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, params=eg.SolverParams(method=method, precond=eg.PREC_ILU0, max_iter=3000, tol=1e-10,
                                             precision=eg.MIXED))
    assert r["info"] == 1 and r["refinements"] == 0  # these methods run in FP64
    assert abs(r["iters"] - r_ref["iters"]) <= 1
    assert rel(x, x_ref) < 1e-8


def test_gcr_maxiter_status(ctx):
    p, _, _, v, b, _ = PROBLEMS["hex8"]()
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, params=eg.SolverParams(method=eg.GCR, precond=eg.PREC_NONE, max_iter=3, tol=1e-14,
                                             abort_not_converged=False))
    assert r["info"] == 2 and r["iters"] == 3


@pytest.mark.parametrize("method", [eg.GCR, eg.BICGSTABL], ids=["gcr", "bicgstabl"])
def test_divergence_tolerance(ctx, method):
    """Linear System Divergence Tolerance (IterSolve.src:364-366): GCR and BiCGStab(l) stop with
    HUTI_DIVERGENCE (3) when the residual ratio exceeds it (IterativeMethods.src:626-629,
    959-961).  A far-off initial guess exceeds a bound of 10 before the first iteration, as in the
    oracle; a bound the decreasing residual never reaches leaves the solve as it was."""
    p, _, _, v, b, _ = PROBLEMS["hex8"]()
    omethod = oracle.GCR if method == eg.GCR else oracle.BICGSTABL
    A = eg.Matrix(ctx, _pat(p), v)
    x0 = np.full(p.n, 100.0)
    x_ref, r_ref = oracle.solve(p, v, b, method=omethod, precond=eg.PREC_DIAGONAL, max_iter=3000, tol=1e-10,
                                x0=x0, divtol=10.0)
    assert r_ref["info"] == 3 and r_ref["iters"] == 0
    x, r = A.solve(b, x0=x0, params=eg.SolverParams(method=method, precond=eg.PREC_DIAGONAL, max_iter=3000, tol=1e-10,
                                                    divtol=10.0, abort_not_converged=False))
    assert r["info"] == 3 and r["iters"] == 0
    assert rel(x, x_ref) < 1e-12
    x_ref, r_ref = oracle.solve(p, v, b, method=omethod, precond=eg.PREC_DIAGONAL, max_iter=3000, tol=1e-10,
                                divtol=1e3)
    x, r = A.solve(b, params=eg.SolverParams(method=method, precond=eg.PREC_DIAGONAL, max_iter=3000, tol=1e-10,
                                             divtol=1e3))
    assert r_ref["info"] == 1 and r["info"] == 1
    assert abs(r["iters"] - r_ref["iters"]) <= 1
    assert rel(x, x_ref) < 1e-8
