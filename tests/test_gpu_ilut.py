"""Threshold ILU (Linear System Preconditioning = ILUT) on the GPU against the oracle.

CRS_ILUT (fem/src/CRSMatrix.src:2849-3044) decides its structure from the values, so the
library factors on the host, as the reference does, and applies the factor on the device
with the same triangular-solve schedules as ILU(n).  The factor must match the oracle's
restatement exactly (structure and bits); the M^-1 application within 1e-13 (bit-exact on
the single-block schedule); solves within one iteration and 1e-8 of the oracle's.
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
    "hex10": lambda: poisson_problem(meshgen.hex_cube(10)),
    "tet8": lambda: poisson_problem(meshgen.tet_cube(8)),
    "elastic4": lambda: elastic_problem(meshgen.hex_cube(4)),
}


@pytest.mark.parametrize("tol", [0.0, 1e-3, 2e-2])
@pytest.mark.parametrize("name", list(PROBLEMS))
def test_ilut_factor_bit_exact(ctx, name, tol):
    p, _, _, v, _, _ = PROBLEMS[name]()
    A = eg.Matrix(ctx, _pat(p), v)
    r, c, d, val = A.ilut(tol, scale_system=True)
    vs = v.copy()
    oracle.scale(p, vs)
    rr, cc, dd, vv = oracle.ilut(p, vs, tol)
    assert np.array_equal(r, rr) and np.array_equal(c, cc) and np.array_equal(d, dd)
    assert np.array_equal(val, vv)
    b = np.random.default_rng(2).standard_normal(p.n)
    u = A.lu_precondition(b)
    assert rel(u, oracle.lusolve_on(rr, cc, dd, vv, b)) < 1e-13


@pytest.mark.parametrize("mode", ["block", "syncfree"])
def test_ilut_apply_each_schedule(ctx, monkeypatch, mode):
    monkeypatch.setenv("EGPU_TRI_MODE", mode)
    p, _, _, v, _, _ = poisson_problem(meshgen.hex_cube(12))
    A = eg.Matrix(ctx, _pat(p), v)
    r, c, d, val = A.ilut(1e-3)
    b = np.random.default_rng(4).standard_normal(p.n)
    u = A.lu_precondition(b)
    ref = oracle.lusolve_on(r, c, d, val, b)
    if mode == "block" and A.tri_info()["single_block_fp64"]:
        assert np.array_equal(u, ref)  # CRS_LUSolve's operation order
    else:
        assert rel(u, ref) < 1e-13


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("method", [eg.BICGSTAB, eg.GCR], ids=["bicgstab", "gcr"])
@pytest.mark.parametrize("name,tol", [("hex10", 1e-3), ("tet8", 1e-2), ("elastic4", 1e-4)])
def test_ilut_solves(ctx, name, tol, method, precision):
    p, _, _, v, b, _ = PROBLEMS[name]()
    stol = 1e-12 if precision == "mixed" else 1e-10
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=oracle.PREC_ILUT, ilut_tol=tol, max_iter=3000,
                                tol=stol)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    prm = eg.SolverParams(method=method, precond=eg.PREC_ILUT, ilut_tol=tol, max_iter=3000, tol=stol,
                          precision=eg.MIXED if precision == "mixed" else eg.FP64)
    x, r = A.solve(b, params=prm)
    assert r["info"] == 1
    if precision == "fp64":
        assert abs(r["iters"] - r_ref["iters"]) <= 1, (r["iters"], r_ref["iters"])
    assert rel(x, x_ref) < 1e-8


def test_ilut_tolerance_change_refactors(ctx):
    """A new ILUT tolerance (or switching to ILU0 and back) rebuilds the factor's structure."""
    p, _, _, v, b, _ = poisson_problem(meshgen.hex_cube(9))
    A = eg.Matrix(ctx, _pat(p), v)
    for pc, tol in ((eg.PREC_ILUT, 1e-2), (eg.PREC_ILUT, 1e-4), (eg.PREC_ILU0, 0.0), (eg.PREC_ILUT, 1e-2)):
        prm = eg.SolverParams(method=eg.BICGSTAB, precond=pc, ilut_tol=tol, max_iter=2000, tol=1e-10,
                              refactorize=False)
        x, r = A.solve(b, params=prm)
        x_ref, r_ref = oracle.solve(p, v, b, method=eg.BICGSTAB, precond=pc, ilut_tol=tol, max_iter=2000, tol=1e-10)
        assert r["info"] == 1 and abs(r["iters"] - r_ref["iters"]) <= 1
        assert rel(x, x_ref) < 1e-8


def test_ilut_refused_for_batches(ctx):
    p, _, _, v, b, _ = poisson_problem(meshgen.hex_cube(4))
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILUT, ilut_tol=1e-3, max_iter=100, tol=1e-8,
                          precision=eg.MIXED)
    with pytest.raises(eg.LibError):
        B = eg.Batch(ctx, prm)
        B.add(_pat(p), v, b)
