"""Device blocks freed by the library are cached and handed out again (csrc/egpu_devmem.h).

A recycled block holds whatever the previous owner left in it: sentinels of a triangular
solve, another system's vectors or factors.  Matrices of changing sizes are created, solved
and freed in turn, so later systems run on recycled blocks of other sizes; every result must
still equal the oracle's, in FP64 and mixed precision, with ILU0 and Jacobi.
"""
import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen
from helpers import poisson_problem, rel

pytestmark = pytest.mark.gpu


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


def test_solves_on_recycled_blocks(ctx):
    problems = {m: poisson_problem(meshgen.hex_cube(m), elem_k=np.exp(np.random.default_rng(m).normal(0, 1, m ** 3)))
                for m in (6, 11, 8, 13)}
    cases = [(eg.BICGSTAB, eg.PREC_ILU0, eg.FP64), (eg.CG, eg.PREC_DIAGONAL, eg.MIXED),
             (eg.BICGSTAB, eg.PREC_ILU0, eg.MIXED)]
    for rnd in range(3):
        for m in ((6, 11, 8, 13), (13, 8, 11, 6), (11, 6, 13, 8))[rnd]:
            p, _, _, v, b, _ = problems[m]
            for method, prec, precision in cases:
                tol = 1e-12 if precision == eg.MIXED else 1e-10
                A = eg.Matrix(ctx, _pat(p), v)
                x, r = A.solve(b, params=eg.SolverParams(method=method, precond=prec, max_iter=2000, tol=tol,
                                                         precision=precision))
                x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=prec, max_iter=2000, tol=tol)
                assert r["info"] == 1 and r_ref["info"] == 1
                if precision == eg.FP64:
                    assert abs(r["iters"] - r_ref["iters"]) <= 1
                assert rel(x, x_ref) < 1e-8
                A.free()


def test_release_cached_memory(ctx):
    """Freed blocks are counted in the cache; releasing gives them back and empties it, and the
    next matrix allocates afresh and still solves like the oracle."""
    p, _, _, v, b, _ = poisson_problem(meshgen.hex_cube(9))
    A = eg.Matrix(ctx, _pat(p), v)
    A.solve(b, params=eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=1e-10))
    A.free()
    held = eg.cached_bytes(ctx.device)
    assert held > 0 and held % (1 << 16) == 0
    assert eg.cached_bytes(-1) >= held
    assert eg.release_cached_memory(ctx.device) == held
    assert eg.cached_bytes(ctx.device) == 0 and eg.release_cached_memory(ctx.device) == 0
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, params=eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=1e-10))
    x_ref, r_ref = oracle.solve(p, v, b, method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=1e-10)
    assert r["info"] == 1 and abs(r["iters"] - r_ref["iters"]) <= 1 and rel(x, x_ref) < 1e-8
    A.free()
