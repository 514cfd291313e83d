"""Mixed-precision BiCGStab + ILU0 with the factors applied by Jacobi sweeps in the FP32 inner
solves (egpu_params.ilu_sweeps): y <- v - L y and z <- D^-1 (y - U z), a fixed number of times
per triangle, instead of exact triangular solves.  The FP64 refinement stops on the true
residual, so every solution meets the tolerance and stays within 1e-8 of the oracle's exact
ILU0 solve (CRS_LUSolve, fem/src/CRSMatrix.src:3346-3363).  ILU(n) with n > 0 and the FP64
drop-in keep the exact solves whatever ilu_sweeps says.
"""
import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
import properties as P
from elmerfem_b200 import meshgen
from helpers import elastic_problem, poisson_problem, rel

pytestmark = pytest.mark.gpu

PROBLEMS = {
    "hex12_lognormal": lambda: poisson_problem(meshgen.hex_cube(12),
                                               elem_k=meshgen.lognormal_conductivity(12 ** 3, 1.0, 7)),
    "tet8": lambda: poisson_problem(meshgen.tet_cube(8)),
    "elastic6": lambda: elastic_problem(meshgen.hex_cube(6)),
    "hex40": lambda: poisson_problem(meshgen.hex_cube(40)),
}


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


@pytest.mark.parametrize("sweeps", [1, 2, 4])
@pytest.mark.parametrize("name", list(PROBLEMS))
def test_sweeps_meet_the_tolerance_against_the_oracle(ctx, monkeypatch, name, sweeps):
    monkeypatch.setenv("EGPU_MIXED_AUTO", "0")
    tol = 1e-10
    p, _, _, v, b, _ = PROBLEMS[name]()
    x_ref, r_ref = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, max_iter=5000, tol=tol)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    try:
        prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=tol, max_iter=5000, precision=eg.MIXED,
                              ilu_sweeps=sweeps)
        x, r = A.solve(b, params=prm)
        assert r["info"] == 1 and r["precision_used"] == eg.MIXED
        assert rel(x, x_ref) < 1e-8
        assert P.scaled_residual(_pat(p), v, b, x) < 1.5 * tol
        # the same matrix again: the sweep layout is rebuilt from the new factors
        x2, r2 = A.solve(b, params=prm)
        assert r2["info"] == 1 and rel(x2, x_ref) < 1e-8
    finally:
        A.free()


def test_exact_paths_ignore_sweeps(ctx, monkeypatch):
    """FP64 drop-in and ILU(1) solve exactly: the same iterations as without ilu_sweeps."""
    monkeypatch.setenv("EGPU_MIXED_AUTO", "0")
    p, _, _, v, b, _ = PROBLEMS["hex12_lognormal"]()
    A = eg.Matrix(ctx, _pat(p), v)
    try:
        for precision, order in ((eg.FP64, 0), (eg.MIXED, 1)):
            base = dict(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=1e-10, max_iter=5000, precision=precision,
                        ilu_order=order)
            x0, r0 = A.solve(b, params=eg.SolverParams(**base))
            x1, r1 = A.solve(b, params=eg.SolverParams(**base, ilu_sweeps=3))
            assert r0["info"] == r1["info"] == 1
            assert r0["iters"] == r1["iters"]
            assert np.array_equal(x0, x1)
    finally:
        A.free()


@pytest.mark.parametrize("sweeps", [1, 2])
def test_batched_sweeps_against_the_oracle(ctx, sweeps):
    """egpu_batch with ilu_sweeps > 0: every system of a mixed batch (hex Poisson with
    log-normal conductivity, and a tet mesh) within 1e-8 of the oracle's exact ILU0 solve."""
    tol = 1e-11
    systems = []
    for i, m in enumerate([6, 11, 8, 5, 9]):
        mesh = meshgen.hex_cube(m) if i % 2 == 0 else meshgen.tet_cube(m)
        k = meshgen.lognormal_conductivity(mesh.nelem, 1.0, 20 + i)
        p, _, _, v, b, _ = poisson_problem(mesh, elem_k=k, load=meshgen.sine_source(mesh.coords))
        systems.append((p, v, b))
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=tol, max_iter=5000, ilu_sweeps=sweeps)
    B = eg.Batch(ctx, prm, chunk=16)
    try:
        ids = [B.add(_pat(p), v, b) for p, v, b in systems]
        B.solve()
        for sid, (p, v, b) in zip(ids, systems):
            r = B.result(sid)
            assert r["info"] == 1, r
            x_ref, r_ref = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, max_iter=5000,
                                        tol=tol)
            assert rel(B.solution(sid), x_ref) < 1e-8
    finally:
        B.free()
