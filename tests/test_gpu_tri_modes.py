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


# ---- node-block sync-free solve: one warp per block of DOF rows (CRS_CreateMatrix with
# DOFs > 1 lays out dense diagonal blocks), levels of the node graph instead of rows

def _random_dof_problem(mesh, dofs, seed=5):
    """A pattern with `dofs` DOFs per node and diagonally dominant random values."""
    p = oracle.create_pattern(mesh, dofs=dofs)
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1.0, 1.0, p.nnz)
    v[p.diag - 1] = np.diff(p.rows).astype(np.float64) + 1.0
    return p, v


NODE_BLOCK_CASES = {
    "elastic5": lambda: elastic_problem(meshgen.hex_cube(5))[::3],
    "elastic8": lambda: elastic_problem(meshgen.hex_cube(8))[::3],
    "tet6_dofs2": lambda: _random_dof_problem(meshgen.tet_cube(6), 2),
    "hex4_dofs4": lambda: _random_dof_problem(meshgen.hex_cube(4), 4),
}


@pytest.mark.parametrize("name", list(NODE_BLOCK_CASES))
def test_node_block_lu_precondition(ctx, monkeypatch, name):
    monkeypatch.setenv("EGPU_TRI_NODE_BLOCKS", "1")
    p, v = NODE_BLOCK_CASES[name]()
    A = eg.Matrix(ctx, _pat(p), v)
    ilu, _ = A.ilu0(scale_system=True)
    vs = v.copy()
    oracle.scale(p, vs)
    ref = oracle.ilu0(p, vs)
    assert np.array_equal(ilu, ref)
    info = A.tri_info()
    assert info["node_block"] == p.dofs
    assert not info["single_block_fp64"] and not info["single_block_fp32"]
    for seed in (3, 4):
        b = np.random.default_rng(seed).standard_normal(p.n)
        u = A.lu_precondition(b)
        assert rel(u, oracle.lusolve(p, ref, b)) < 1e-13


def test_node_block_levels(ctx, monkeypatch):
    """Blocks of 3 elasticity DOFs: about a third of the row levels; off when disabled."""
    p, _, _, v, _, _ = elastic_problem(meshgen.hex_cube(8))
    monkeypatch.setenv("EGPU_TRI_NODE_BLOCKS", "0")
    A = eg.Matrix(ctx, _pat(p), v)
    A.ilu0()
    rows = A.tri_info()
    monkeypatch.setenv("EGPU_TRI_NODE_BLOCKS", "1")
    B = eg.Matrix(ctx, _pat(p), v)
    B.ilu0()
    blk = B.tri_info()
    assert rows["node_block"] == 1 and blk["node_block"] == 3
    assert blk["lower_levels"] * 2 < rows["lower_levels"]
    assert blk["upper_levels"] * 2 < rows["upper_levels"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("method", [eg.BICGSTAB, eg.GCR, eg.BICGSTABL], ids=["bicgstab", "gcr", "bicgstabl"])
@pytest.mark.parametrize("name", ["elastic5", "elastic8"])
def test_node_block_solves(ctx, monkeypatch, name, method, precision):
    monkeypatch.setenv("EGPU_TRI_NODE_BLOCKS", "1")
    p, _, _, v, b, _ = elastic_problem(meshgen.hex_cube(5 if name == "elastic5" else 8))
    tol = 1e-12 if precision == "mixed" else 1e-10
    extra = {"restart": 4} if method == eg.BICGSTABL else {}
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=eg.PREC_ILU0, max_iter=3000, tol=tol, **extra)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    prm = eg.SolverParams(method=method, precond=eg.PREC_ILU0, max_iter=3000, tol=tol,
                          precision=eg.MIXED if precision == "mixed" else eg.FP64, **extra)
    x, r = A.solve(b, params=prm)
    assert r["info"] == 1
    assert A.tri_info()["node_block"] == 3
    if precision == "fp64":
        assert abs(r["iters"] - r_ref["iters"]) <= 1, (r["iters"], r_ref["iters"])
    assert rel(x, x_ref) < 1e-8


def test_node_block_lu_precondition_elastic32(ctx, monkeypatch):
    """3-DOF elasticity 32^3 (107,811 rows) on the schedule the cost model picks by itself (node
    blocks); also the case the node-block apply profile is captured on."""
    monkeypatch.delenv("EGPU_TRI_NODE_BLOCKS", raising=False)
    monkeypatch.delenv("EGPU_TRI_MODE", raising=False)
    p, _, _, v, _, _ = elastic_problem(meshgen.hex_cube(32))
    A = eg.Matrix(ctx, _pat(p), v)
    ilu, _ = A.ilu0(scale_system=True)
    assert A.tri_info()["node_block"] == 3
    vs = v.copy()
    oracle.scale(p, vs)
    ref = oracle.ilu0(p, vs)
    assert np.array_equal(ilu, ref)
    b = np.random.default_rng(7).standard_normal(p.n)
    u = A.lu_precondition(b)
    assert rel(u, oracle.lusolve(p, ref, b)) < 1e-13
