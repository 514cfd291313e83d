"""GPU parity through the C ABI against the oracle (needs a B200).

Tolerances of the path: CRS pattern bit-exact; Values within 1e-13 of the row
scale; SpMV within 1e-14 of the row's |a||x| scale; converged solutions within 1e-8
relative of the oracle's at the same tolerance.  ILU0 factors are bit-exact.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import _lib, meshgen
from helpers import renumbered, elastic_problem, poisson_problem, rel, row_rel_max

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _heateq():
    d = np.load(os.path.join(GOLDEN, "heateq_mesh.npz"))
    return meshgen.Mesh(d["coords"], 303, d["elements"], 202, d["bnd_elements"], d["bnd_ids"], ())


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


def test_spmv(ctx):
    m = meshgen.hex_cube(14)
    p, vals, *_ = poisson_problem(m, elem_k=meshgen.lognormal_conductivity(m.nelem, 1.0, 3))
    A = eg.Matrix(ctx, _pat(p), vals)
    u = np.random.default_rng(1).standard_normal(p.n)
    v = A.mv(u)
    ref = oracle.spmv(p, vals, u)
    scale = oracle.spmv(p, np.abs(vals), np.abs(u))
    assert np.max(np.abs(v - ref) / scale) < 1e-14


def test_matvec_subr_hook(ctx):
    m = meshgen.tet_cube(5)
    p, vals, *_ = poisson_problem(m)
    u = np.random.default_rng(2).standard_normal(p.n)
    v = np.zeros(p.n)
    h = C.c_void_p()
    n = C.c_int(p.n)
    zero = C.c_int(0)
    _lib.lib().egpu_matvec_subr(C.byref(h), C.byref(n), p.rows, p.cols, vals, u, v, C.byref(zero))
    assert h.value and zero.value == 0
    assert rel(v, oracle.spmv(p, vals, u)) < 1e-14
    vals2 = vals * 2.0
    _lib.lib().egpu_matvec_subr(C.byref(h), C.byref(n), p.rows, p.cols, vals2, u, v, C.byref(zero))
    assert rel(v, 2.0 * oracle.spmv(p, vals, u)) < 1e-14


@pytest.mark.parametrize("mk", [lambda: meshgen.hex_cube(9), lambda: meshgen.tet_cube(7), _heateq])
def test_ilu0_factor_bit_exact(ctx, mk):
    m = mk()
    p, _, _, v, _, _ = poisson_problem(m)
    A = eg.Matrix(ctx, _pat(p), v)
    ilu, D = A.ilu0(scale_system=True)
    vs = v.copy()
    Dref, _ = oracle.scale(p, vs)
    assert np.array_equal(D, Dref)
    ref = oracle.ilu0(p, vs)
    assert np.array_equal(ilu, ref)
    b = np.random.default_rng(3).standard_normal(p.n)
    u = A.lu_precondition(b)
    assert rel(u, oracle.lusolve(p, ref, b)) < 1e-13


def test_ilu0_elastic_bit_exact(ctx):
    p, _, _, v, _, _ = elastic_problem(meshgen.hex_cube(4))
    A = eg.Matrix(ctx, _pat(p), v)
    ilu, _ = A.ilu0(scale_system=True)
    vs = v.copy()
    oracle.scale(p, vs)
    assert np.array_equal(ilu, oracle.ilu0(p, vs))


@pytest.mark.parametrize("kind", ["hex", "tet", "heateq", "hex_lognormal", "hex_renumbered", "tet_renumbered"])
@pytest.mark.parametrize("sym", [False, True])
def test_assembly_and_dirichlet(ctx, kind, sym):
    if kind == "heateq":
        m, k, load = _heateq(), None, None
    elif kind == "hex_renumbered":  # random node numbering: the bandwidth optimisation is accepted
        m, k, load = renumbered(meshgen.hex_cube(6), 1), None, None
    elif kind == "tet_renumbered":
        m, k, load = renumbered(meshgen.tet_cube(5), 2), None, None
    elif kind == "hex":
        m, k, load = meshgen.hex_cube(7), None, None
    elif kind == "tet":
        m, k, load = meshgen.tet_cube(6), None, None
    else:
        m = meshgen.hex_cube(8)
        k, load = meshgen.lognormal_conductivity(m.nelem, 1.0, 1), meshgen.sine_source(m.coords)
    p, vals0, rhs0, v, b, con = poisson_problem(m, elem_k=k, load=load, sym=sym)
    pp = eg.create_matrix(m)
    assert np.array_equal(pp.cols, p.cols)
    A = eg.Matrix(ctx, pp)
    A.bind_assembly(m)
    A.assemble_poisson(elem_k=k, nodal_k=None if k is not None else np.ones(m.nnodes),
                       load=np.ones(m.nnodes) if load is None else load)
    assert row_rel_max(p, A.values(), vals0) < 1e-13
    assert rel(A.rhs(), rhs0) < 1e-13
    A.dirichlet(con, symmetric=sym)
    assert row_rel_max(p, A.values(), v) < 1e-13
    assert np.max(np.abs(A.rhs() - b)) <= 1e-13 * np.max(np.abs(b))


def test_elastic_assembly(ctx):
    m = meshgen.hex_cube(4)
    p, vals0, rhs0, v, b, con = elastic_problem(m)
    pp = eg.create_matrix(m, dofs=3)
    A = eg.Matrix(ctx, pp)
    A.bind_assembly(m)
    A.assemble_elastic(200e9, 0.3, (0.0, 0.0, -1e4))
    assert row_rel_max(p, A.values(), vals0) < 1e-13
    assert rel(A.rhs(), rhs0) < 1e-13
    A.dirichlet(con)
    assert row_rel_max(p, A.values(), v) < 1e-13


CASES = [
    ("hex10_bicgstab_ilu0", lambda: poisson_problem(meshgen.hex_cube(10)), eg.BICGSTAB, eg.PREC_ILU0),
    ("hex10_cg_ilu0", lambda: poisson_problem(meshgen.hex_cube(10)), eg.CG, eg.PREC_ILU0),
    ("hex12_cg_jacobi_lognormal", lambda: poisson_problem(
        meshgen.hex_cube(12), elem_k=meshgen.lognormal_conductivity(12 ** 3, 1.0, 1),
        load=meshgen.sine_source(meshgen.hex_cube(12).coords), sym=True), eg.CG, eg.PREC_DIAGONAL),
    ("tet8_cg_jacobi", lambda: poisson_problem(meshgen.tet_cube(8), sym=True), eg.CG, eg.PREC_DIAGONAL),
    ("tet8_bicgstab_none", lambda: poisson_problem(meshgen.tet_cube(8)), eg.BICGSTAB, eg.PREC_NONE),
    ("tet8_bicgstab_jacobi", lambda: poisson_problem(meshgen.tet_cube(8)), eg.BICGSTAB, eg.PREC_DIAGONAL),
    ("elastic5_bicgstab_ilu0", lambda: elastic_problem(meshgen.hex_cube(5)), eg.BICGSTAB, eg.PREC_ILU0),
    ("hex9_renumbered_bicgstab_ilu0", lambda: poisson_problem(renumbered(meshgen.hex_cube(9), 3)), eg.BICGSTAB,
     eg.PREC_ILU0),
    ("tet7_renumbered_cg_jacobi", lambda: poisson_problem(renumbered(meshgen.tet_cube(7), 4), sym=True), eg.CG,
     eg.PREC_DIAGONAL),
]


@pytest.mark.parametrize("name,make,method,prec", CASES, ids=[c[0] for c in CASES])
def test_fp64_solve_matches_oracle(ctx, name, make, method, prec):
    p, _, _, v, b, _ = make()
    tol = 1e-10
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=prec, max_iter=2000, tol=tol)
    assert r_ref["info"] == 1
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, params=eg.SolverParams(method=method, precond=prec, max_iter=2000, tol=tol))
    assert r["info"] == 1
    assert abs(r["iters"] - r_ref["iters"]) <= 1, (r["iters"], r_ref["iters"])
    assert rel(x, x_ref) < 1e-8


@pytest.mark.parametrize("name,make,method,prec", CASES, ids=[c[0] for c in CASES])
def test_mixed_solve_matches_oracle(ctx, name, make, method, prec):
    p, _, _, v, b, _ = make()
    x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=prec, max_iter=4000, tol=1e-12)
    A = eg.Matrix(ctx, _pat(p), v)
    prm = eg.SolverParams(method=method, precond=prec, max_iter=4000, tol=1e-12, precision=eg.MIXED)
    x, r = A.solve(b, params=prm)
    assert r["info"] == 1 and r["refinements"] >= 1
    assert rel(x, x_ref) < 1e-8


def test_heateq_nrm_on_gpu(ctx):
    """fem/tests/heateq (a.sif: BiCGStab + ILU0, tol 1e-8): assembled and solved on the GPU."""
    t = json.load(open(os.path.join(GOLDEN, "targets.json")))["heateq"]
    m = _heateq()
    pp = eg.create_matrix(m)
    A = eg.Matrix(ctx, pp)
    A.bind_assembly(m, cdim=2)
    A.assemble_poisson(nodal_k=np.ones(m.nnodes), load=np.ones(m.nnodes))
    con = np.sort(pp.perm[m.boundary_nodes(range(1, 7)) - 1])
    A.dirichlet(con)
    x, r = A.solve(params=eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=350, tol=1e-8))
    nrm = eg.compute_norm(x)
    assert abs(nrm - t["nrm"]) / t["nrm"] < t["eps"]
    x, r = A.solve(params=eg.SolverParams(method=eg.CG, precond=eg.PREC_ILU0, max_iter=350, tol=1e-12))
    assert abs(eg.compute_norm(x) - t["nrm"]) / t["nrm"] < 1e-9


@pytest.mark.parametrize("case,method", [(5, eg.CG), (10, eg.BICGSTAB)])
def test_linearsolvers_nrm_on_gpu(ctx, case, method):
    m = _heateq()
    pp = eg.create_matrix(m)
    A = eg.Matrix(ctx, pp)
    A.bind_assembly(m, cdim=2)
    A.assemble_poisson(nodal_k=np.ones(m.nnodes), load=None)
    con = np.sort(pp.perm[m.boundary_nodes(range(1, 7)) - 1])
    A.dirichlet(con, np.full(con.size, float(case)))
    x, r = A.solve(params=eg.SolverParams(method=method, precond=eg.PREC_ILU0, max_iter=3500, tol=1e-12))
    assert abs(eg.compute_norm(x) - case) / case < 1e-9


def test_zero_rhs_and_maxiter(ctx):
    p, _, _, v, b, _ = poisson_problem(meshgen.hex_cube(6))
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(np.zeros(p.n), params=eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, max_iter=5))
    assert r["info"] == 1 and not np.any(x)
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, max_iter=3, tol=1e-14, abort_not_converged=False)
    x, r = A.solve(b, params=prm)
    x_ref, r_ref = oracle.solve(p, v, b, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=3, tol=1e-14)
    assert r["info"] == r_ref["info"] == 2 and r["iters"] == r_ref["iters"] == 4
    assert rel(x, x_ref) < 1e-12
    with pytest.raises(eg.NotConverged):
        A.solve(b, params=eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, max_iter=3, tol=1e-14))


def test_nonzero_initial_guess(ctx):
    p, _, _, v, b, _ = poisson_problem(meshgen.tet_cube(6))
    x0 = np.random.default_rng(5).random(p.n)
    x_ref, r_ref = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, max_iter=500, tol=1e-10,
                                x0=x0)
    A = eg.Matrix(ctx, _pat(p), v)
    x, r = A.solve(b, x0=x0, params=eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=500, tol=1e-10))
    assert abs(r["iters"] - r_ref["iters"]) <= 1 and rel(x, x_ref) < 1e-8
