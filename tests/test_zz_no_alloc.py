"""The allocation-free CG entry point (egpu_cg_noalloc) against the regular one.

Callers whose device memory belongs to another runtime, or that cannot afford the implicit
synchronisation of cudaMalloc inside their loop, cannot let the library allocate.  For them
egpu_cg_noalloc keeps all scratch in one fixed device array inside the library.  This test
calls it through the C ABI twice in a row on the caller's device arrays and checks each
result against egpu_iter_solve_dev (the entry point that allocates its workspace) with the
tolerance the other solve tests use: solution within 1e-8 relative, same HUTI status and
iteration count within one.  It lives in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

import elmerfem_b200 as eg
from elmerfem_b200 import _lib, meshgen
from helpers import poisson_problem, rel

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("mesh,prec", [(lambda: meshgen.hex_cube(11), eg.PREC_DIAGONAL),
                                       (lambda: meshgen.tet_cube(30), eg.PREC_DIAGONAL),
                                       (lambda: meshgen.hex_cube(9), eg.PREC_NONE)])
def test_noalloc_matches_allocating_entry_point(ctx, mesh, prec):
    torch = pytest.importorskip("torch")
    m = mesh()
    k = meshgen.lognormal_conductivity(m.nelem, 1.0, 7)
    p, _, _, v, b, _ = poisson_problem(m, elem_k=k, load=meshgen.sine_source(m.coords), sym=True)
    assert p.n <= 32768
    prm = eg.SolverParams(method=eg.CG, precond=prec, max_iter=3000, tol=1e-10)
    A = eg.Matrix(ctx, eg.CRSPattern(p.n, p.nnz, 1, p.perm, p.rows, p.cols, p.diag), v)
    x_ref, r_ref = A.solve(b, params=prm)

    rows, cols, diag = _dev(torch, p.rows), _dev(torch, p.cols), _dev(torch, p.diag)
    vals, bd = _dev(torch, v), _dev(torch, b)
    for _ in range(2):  # the scratch array keeps the previous call's contents
        x = torch.zeros(p.n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        res = _lib.Result()
        cp = prm.to_c()
        rc = _lib.lib().egpu_cg_noalloc(0, p.n, rows.data_ptr(), cols.data_ptr(), diag.data_ptr(), vals.data_ptr(),
                                        bd.data_ptr(), x.data_ptr(), C.byref(cp), C.byref(res))
        assert rc == r_ref["info"] == 1
        assert abs(res.iters - r_ref["iters"]) <= 1
        assert rel(x.cpu().numpy(), x_ref) < 1e-8


def test_noalloc_rejects_systems_beyond_its_limit():
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL).to_c()
    one = C.c_void_p(1)
    rc = _lib.lib().egpu_cg_noalloc(0, 32769, one, one, one, one, one, one, C.byref(prm), None)
    assert rc == -1
    bad = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0).to_c()
    assert _lib.lib().egpu_cg_noalloc(0, 10, one, one, one, one, one, one, C.byref(bad), None) == -1


def test_noalloc_refuses_malformed_arrays(ctx):
    """The caller's arrays are used in place, so the entry point checks them on the device before
    any gather: a Cols entry of n + 1 (one past the last row) and a Diag that does not point at
    its row's diagonal each return EGPU_ERR_ARG, and x is left untouched.  A well-formed call
    afterwards still solves (the error flag does not stick)."""
    torch = pytest.importorskip("torch")
    m = meshgen.hex_cube(5)
    p, _, _, v, b, _ = poisson_problem(m, sym=True)
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, max_iter=500, tol=1e-10)
    rows, vals, bd = _dev(torch, p.rows), _dev(torch, v), _dev(torch, b)
    bad_cols = p.cols.copy()
    bad_cols[p.rows[3] - 1] = p.n + 1
    bad_diag = p.diag.copy()
    bad_diag[4] += 1
    cases = [(_dev(torch, bad_cols), _dev(torch, p.diag)), (_dev(torch, p.cols), _dev(torch, bad_diag))]
    for cols, diag in cases:
        x = torch.full((p.n,), 7.0, dtype=torch.float64, device="cuda")
        cp = prm.to_c()
        rc = _lib.lib().egpu_cg_noalloc(0, p.n, rows.data_ptr(), cols.data_ptr(), diag.data_ptr(), vals.data_ptr(),
                                        bd.data_ptr(), x.data_ptr(), C.byref(cp), None)
        assert rc == -1
        assert bool((x == 7.0).all())
    cols, diag = _dev(torch, p.cols), _dev(torch, p.diag)
    x = torch.zeros(p.n, dtype=torch.float64, device="cuda")
    cp = prm.to_c()
    rc = _lib.lib().egpu_cg_noalloc(0, p.n, rows.data_ptr(), cols.data_ptr(), diag.data_ptr(), vals.data_ptr(),
                                    bd.data_ptr(), x.data_ptr(), C.byref(cp), None)
    assert rc == 1
