"""ILU(n) (Linear System Preconditioning = ILU1, ILU2, ...) on the GPU against the oracle.

CRS_IncompleteLU(A, n) (CRSMatrix.src:2157-2500) factors on the structure InitializeILU1
builds n times.  The device factors must equal the oracle's restatement bit for bit (same
structure, same IKJ order), the preconditioner apply must match, and solves must agree with
the oracle's (iterations within 1, solution within 1e-8).
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
    "hex8": lambda: poisson_problem(meshgen.hex_cube(8)),
    "tet6": lambda: poisson_problem(meshgen.tet_cube(6)),
    "heateq": lambda: poisson_problem(_heateq()),
    "elastic3": lambda: elastic_problem(meshgen.hex_cube(3)),
    "hex16_lognormal": lambda: poisson_problem(meshgen.hex_cube(16), elem_k=meshgen.lognormal_conductivity(16 ** 3, 1.0, 3)),
}


@pytest.mark.parametrize("mode", ["block", "syncfree"])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("name", ["hex8", "tet6", "heateq", "elastic3"])
def test_iluk_factors_bit_exact(ctx, monkeypatch, mode, order, name):
    monkeypatch.setenv("EGPU_TRI_MODE", mode)
    p, _, _, v, _, _ = PROBLEMS[name]()
    A = eg.Matrix(ctx, _pat(p), v)
    r, c, d, f = A.ilu(order, scale_system=True)
    vs = v.copy()
    oracle.scale(p, vs)
    rr, cr, dr, fr = oracle.iluk(p, vs, order)
    assert np.array_equal(r, rr) and np.array_equal(c, cr) and np.array_equal(d, dr)
    assert np.array_equal(f, fr)
    # M^-1 with the ILU(n) factors (CRS_LUSolve on the ILU structure)
    q = oracle.Pattern(p.n, cr.size, p.dofs, p.perm, rr, cr, dr, 0, 0, 0, 0)
    b = np.random.default_rng(order).standard_normal(p.n)
    u = A.lu_precondition(b)
    ref = oracle.lusolve(q, fr, b)
    if mode == "block":
        assert np.array_equal(u, ref)  # the single-block solve keeps CRS_LUSolve's operation order
    else:
        assert rel(u, ref) < 1e-13


@pytest.mark.parametrize("mode", ["block", "syncfree"])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("method", [eg.BICGSTAB, eg.CG], ids=["bicgstab", "cg"])
@pytest.mark.parametrize("name", ["hex8", "elastic3", "hex16_lognormal"])
def test_iluk_fp64_solve_matches_oracle(ctx, monkeypatch, mode, order, method, name):
    if method == eg.CG and name == "elastic3":
        pytest.skip("the elasticity system is solved with BiCGStab")
    monkeypatch.setenv("EGPU_TRI_MODE", mode)
    p, _, _, v, b, _ = PROBLEMS[name]()
    tol = 1e-10
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=eg.PREC_ILU0, max_iter=2000, tol=tol, ilu_order=order)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    prm = eg.SolverParams(method=method, precond=eg.PREC_ILU0, ilu_order=order, max_iter=2000, tol=tol)
    x, r = A.solve(b, params=prm)
    assert r["info"] == 1
    assert abs(r["iters"] - r_ref["iters"]) <= 1, (r["iters"], r_ref["iters"])
    assert rel(x, x_ref) < 1e-8


@pytest.mark.parametrize("order", [1, 2])
def test_iluk_mixed_and_order_switch(ctx, order):
    """Mixed precision with ILU(n); the same matrix re-factored at another order."""
    p, _, _, v, b, _ = PROBLEMS["hex16_lognormal"]()
    x_ref, _ = oracle.solve(p, v, b, method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=4000, tol=1e-12)
    A = eg.Matrix(ctx, _pat(p), v)
    for k in (order, 0, order):
        prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, ilu_order=k, max_iter=4000, tol=1e-12,
                              precision=eg.MIXED)
        x, r = A.solve(b, params=prm)
        assert r["info"] == 1
        assert rel(x, x_ref) < 1e-8


def test_iluk_batch(ctx):
    """Batched mixed solves with ILU1 against the oracle's FP64 ILU1 solutions."""
    sizes = [4, 6, 8, 5]
    systems = []
    for i, m in enumerate(sizes):
        mesh = meshgen.hex_cube(m)
        p, _, _, v, b, _ = poisson_problem(mesh, elem_k=meshgen.lognormal_conductivity(mesh.nelem, 1.0, 20 + i))
        systems.append((p, v, b))
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, ilu_order=1, tol=1e-11, max_iter=5000)
    B = eg.Batch(ctx, prm, chunk=16)
    ids = [B.add(_pat(p), v, b) for p, v, b in systems]
    B.solve()
    for sid, (p, v, b) in zip(ids, systems):
        assert B.result(sid)["info"] == 1
        x_ref, _ = oracle.solve(p, v, b, method=eg.BICGSTAB, precond=eg.PREC_ILU0, ilu_order=1, max_iter=5000,
                                tol=1e-11)
        assert rel(B.solution(sid), x_ref) < 1e-8
    B.free()
