"""The two single-system workloads at their full sizes on the device, checked through
size-independent properties (tests/properties.py) where the oracle would take minutes:

* Poisson on the 128^3 hex mesh (2,146,689 rows, 57.1 M nonzeros), log-normal element
  conductivity (sigma 1, seed 1): the assembled matrix annihilates constants, is symmetric and
  integrates the energy of a linear field to sum_e k_e vol_e; a unit load integrates to the
  volume; the device SpMV agrees with a host product; with the sine source and symmetric zero
  Dirichlet conditions, CG + Diagonal in FP64 and in mixed precision both meet the scaled
  stopping test (1e-10) and agree within 1e-8.
* Elasticity on the 64^3 hex mesh (823,875 rows, 64.7 M nonzeros): the matrix annihilates the
  six rigid-body modes and is symmetric, the body force integrates to force x volume; clamped
  at x = 0, BiCGStab + ILU0 in FP64 and mixed precision meet the stopping test (1e-8) and agree
  within 1e-8.
"""
import numpy as np
import pytest

import elmerfem_b200 as eg
import properties as P
from elmerfem_b200 import meshgen
from helpers import rel

pytestmark = pytest.mark.gpu


def test_poisson_hex128_lognormal(ctx):
    m = meshgen.hex_cube(128)
    k = meshgen.lognormal_conductivity(m.nelem, 1.0, 1)
    pat = eg.create_matrix(m)
    assert (pat.n, pat.nnz) == (129 ** 3, 385 ** 3)
    A = eg.Matrix(ctx, pat)
    try:
        A.bind_assembly(m)
        A.assemble_poisson(elem_k=k, load=np.ones(m.nnodes))
        vals, rhs = A.values(), A.rhs()
        assert P.row_sum_defect(pat, vals) < 1e-12
        assert P.symmetry_defect(pat, vals) < 1e-13
        assert P.linear_field_energy_defect(m, pat, vals, k) < 1e-11
        assert abs(rhs.sum() - 1.0) < 1e-11
        u = np.random.default_rng(5).standard_normal(pat.n)
        assert rel(A.mv(u), P.csr(pat, vals) @ u) < 1e-14

        A.assemble_poisson(elem_k=k, load=meshgen.sine_source(m.coords))
        con = np.sort(pat.perm[m.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)
        A.dirichlet(con, symmetric=True)
        v, b = A.values(), A.rhs()
        assert P.symmetry_defect(pat, v) < 1e-13
        tol = 1e-10
        x64, r64 = A.solve(b, params=eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=tol,
                                                     max_iter=20000))
        xm, rm = A.solve(b, params=eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=tol,
                                                   max_iter=20000, precision=eg.MIXED))
        assert r64["info"] == 1 and rm["info"] == 1
        assert P.scaled_residual(pat, v, b, x64) < 1.5 * tol
        assert P.scaled_residual(pat, v, b, xm) < 1.5 * tol
        assert rel(xm, x64) < 1e-8
    finally:
        A.free()


def test_elasticity_hex64(ctx):
    m = meshgen.hex_cube(64)
    pat = eg.create_matrix(m, dofs=3)
    assert (pat.n, pat.nnz) == (3 * 65 ** 3, 9 * 193 ** 3)
    A = eg.Matrix(ctx, pat)
    force = (0.0, 0.0, -1e4)
    try:
        A.bind_assembly(m)
        A.assemble_elastic(200e9, 0.3, force)
        vals, rhs = A.values(), A.rhs()
        assert P.rigid_mode_defect(m, pat, vals) < 1e-10
        assert P.symmetry_defect(pat, vals) < 1e-13
        for d in range(3):  # row 3 (Perm(node) - 1) + d holds component d
            assert abs(rhs[d::3].sum() - force[d]) < 1e-10 * 1e4

        nodes = pat.perm[m.boundary_nodes([1]) - 1]
        con = np.sort(np.concatenate([3 * (nodes - 1) + d for d in (1, 2, 3)])).astype(np.int32)
        A.dirichlet(con, symmetric=False)
        v, b = A.values(), A.rhs()
        tol = 1e-8
        x64, r64 = A.solve(b, params=eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=tol,
                                                     max_iter=20000))
        xm, rm = A.solve(b, params=eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=tol,
                                                   max_iter=20000, precision=eg.MIXED))
        assert r64["info"] == 1 and rm["info"] == 1
        assert P.scaled_residual(pat, v, b, x64) < 1.5 * tol
        assert P.scaled_residual(pat, v, b, xm) < 1.5 * tol
        assert rel(xm, x64) < 1e-8
    finally:
        A.free()
