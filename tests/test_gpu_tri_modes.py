"""Both ILU0 triangular-solve schedules on the GPU, forced one at a time.

EGPU_TRI_MODE=block runs the level-synchronous single-block solve (block 0 of the
persistent kernel, shared-memory ring, cp.async staging); EGPU_TRI_MODE=syncfree the
grid-wide sync-free solve.  The schedule is chosen when a matrix builds its level
schedule, so each test sets the mode before creating its matrix.  The block solve keeps
CRS_LUSolve's operation order (fem/src/CRSMatrix.src:3346-3363), so its FP64 M^-1
application is bit-identical to the oracle's.
"""
import os

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen
from helpers import elastic_problem, poisson_problem, rel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


def _heateq():
    d = np.load(os.path.join(GOLDEN, "heateq_mesh.npz"))
    return meshgen.Mesh(d["coords"], 303, d["elements"], 202, d["bnd_elements"], d["bnd_ids"], ())


PROBLEMS = {
    "hex10": lambda: poisson_problem(meshgen.hex_cube(10)),
    "tet9": lambda: poisson_problem(meshgen.tet_cube(9)),
    "heateq": lambda: poisson_problem(_heateq()),
    "elastic5": lambda: elastic_problem(meshgen.hex_cube(5)),
    "hex32": lambda: poisson_problem(meshgen.hex_cube(32)),
}


@pytest.mark.parametrize("name", ["hex10", "tet9", "heateq", "elastic5", "hex32"])
def test_block_lu_precondition_bit_exact(ctx, monkeypatch, name):
    monkeypatch.setenv("EGPU_TRI_MODE", "block")
    p, _, _, v, _, _ = PROBLEMS[name]()
    A = eg.Matrix(ctx, _pat(p), v)
    ilu, _ = A.ilu0(scale_system=True)
    vs = v.copy()
    oracle.scale(p, vs)
    ref = oracle.ilu0(p, vs)
    assert np.array_equal(ilu, ref)
    for seed in (3, 4):
        b = np.random.default_rng(seed).standard_normal(p.n)
        u = A.lu_precondition(b)
        assert np.array_equal(u, oracle.lusolve(p, ref, b))


@pytest.mark.parametrize("mode", ["block", "syncfree"])
@pytest.mark.parametrize("name", ["hex10", "tet9", "elastic5", "hex32"])
@pytest.mark.parametrize("method", [eg.CG, eg.BICGSTAB], ids=["cg", "bicgstab"])
def test_fp64_ilu0_solve_each_mode(ctx, monkeypatch, mode, name, method):
    monkeypatch.setenv("EGPU_TRI_MODE", mode)
    p, _, _, v, b, _ = PROBLEMS[name]()
    if method == eg.CG and name == "elastic5":
        pytest.skip("the elasticity system is solved with BiCGStab")
    tol = 1e-10
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=eg.PREC_ILU0, max_iter=2000, tol=tol)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, params=eg.SolverParams(method=method, precond=eg.PREC_ILU0, max_iter=2000, tol=tol))
    assert r["info"] == 1
    assert abs(r["iters"] - r_ref["iters"]) <= 1, (r["iters"], r_ref["iters"])
    assert rel(x, x_ref) < 1e-8


@pytest.mark.parametrize("mode", ["block", "syncfree"])
@pytest.mark.parametrize("name", ["hex10", "elastic5", "hex32"])
def test_mixed_ilu0_solve_each_mode(ctx, monkeypatch, mode, name):
    monkeypatch.setenv("EGPU_TRI_MODE", mode)
    p, _, _, v, b, _ = PROBLEMS[name]()
    x_ref, r_ref = oracle.solve(p, v, b, method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=4000, tol=1e-12)
    A = eg.Matrix(ctx, _pat(p), v)
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=4000, tol=1e-12, precision=eg.MIXED)
    x, r = A.solve(b, params=prm)
    assert r["info"] == 1
    assert rel(x, x_ref) < 1e-8


def test_modes_agree_on_clones(ctx, monkeypatch):
    """A clone shares its prototype's block schedule and holds its own factor values."""
    monkeypatch.setenv("EGPU_TRI_MODE", "block")
    p, _, _, v, b, _ = poisson_problem(meshgen.hex_cube(12))
    A = eg.Matrix(ctx, _pat(p), v)
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=2000, tol=1e-10)
    x0, r0 = A.solve(b, params=prm)
    B = eg.Matrix.clone(A)
    B.update_values(2.0 * v)
    x1, r1 = B.solve(b, params=prm)
    assert r0["info"] == 1 and r1["info"] == 1
    assert rel(2.0 * x1, x0) < 1e-8
