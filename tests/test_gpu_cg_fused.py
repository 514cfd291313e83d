"""The FP32 inner CG folds the direction update P = Z + beta P into its SpMV (each gathered
column forms Z + beta P_old with the same fused multiply-add as the separate pass), so the
iterates are bit-identical to the unfused form (EGPU_CG_FUSE=0): same inner iterations,
refinements and solution, with and without Jacobi on a non-unit diagonal, and across
resumed segments (P alternates between two work vectors and the carried one is tracked)."""
import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen
from helpers import poisson_problem, rel

pytestmark = pytest.mark.gpu


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


@pytest.mark.parametrize("scale", [True, False], ids=["scaled", "unscaled"])
@pytest.mark.parametrize("precond", [eg.PREC_DIAGONAL, eg.PREC_NONE], ids=["jacobi", "none"])
@pytest.mark.parametrize("mesh", ["hex20", "tet12"])
def test_fused_direction_update_is_bit_identical(ctx, monkeypatch, mesh, precond, scale):
    monkeypatch.setenv("EGPU_MIXED_AUTO", "0")
    m = meshgen.hex_cube(20) if mesh == "hex20" else meshgen.tet_cube(12)
    p, _, _, v, b, _ = poisson_problem(m, elem_k=meshgen.lognormal_conductivity(m.nelem, 1.0, 5), sym=True)
    prm = eg.SolverParams(method=eg.CG, precond=precond, tol=1e-11, max_iter=5000, precision=eg.MIXED,
                          scale_system=scale, inner_tol=1e-2)
    A = eg.Matrix(ctx, _pat(p), v)
    try:
        x1, r1 = A.solve(b, params=prm)
        monkeypatch.setenv("EGPU_CG_FUSE", "0")
        x0, r0 = A.solve(b, params=prm)
        monkeypatch.delenv("EGPU_CG_FUSE")
        assert r0["info"] == r1["info"] == 1
        assert r0["refinements"] > 1  # resumed segments are covered
        assert (r0["iters"], r0["refinements"]) == (r1["iters"], r1["refinements"])
        assert np.array_equal(x0, x1)
        x_ref, _ = oracle.solve(p, v, b, method=oracle.CG, precond=precond, max_iter=5000, tol=1e-11, scale=scale)
        assert rel(x1, x_ref) < 1e-8
    finally:
        A.free()
