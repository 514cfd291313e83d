"""Failure detection on the device without a fault (needs a B200).

Every device-side wait of the library is bounded by the context's wait limit; a wait that runs
out records EGPU_ERR_TIMEOUT, the kernel returns and the host reads the status, so the context
stays usable.  These tests make a wait run out by design (a grid barrier one block never
reaches, a value nothing publishes) with a 1 ms limit, and cancel a running solve through the
host-mapped abort word.  Nothing here traps, faults or waits without a bound: the reference's
counterpart is only IterSolver's status exits (IterSolve.src:784-792).
"""
import threading
import time

import numpy as np
import pytest

import elmerfem_b200 as eg
from elmerfem_b200 import _lib, meshgen
from helpers import poisson_problem, rel

pytestmark = pytest.mark.gpu


def _small_system(ctx):
    m = meshgen.hex_cube(8)
    p, _, _, v, b, _ = poisson_problem(m, sym=True)
    A = eg.Matrix(ctx, eg.CRSPattern(p.n, p.nnz, 1, p.perm, p.rows, p.cols, p.diag), v)
    return p, v, b, A


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_runs_out_and_context_recovers(ctx, which):
    import oracle

    p, v, b, A = _small_system(ctx)
    try:
        ctx.set_wait_limit(1e-3)
        t0 = time.perf_counter()
        rc = ctx.wait_selftest(which)
        dt = time.perf_counter() - t0
        assert rc == -4  # EGPU_ERR_TIMEOUT
        assert dt < 1.0
        ctx.set_wait_limit(0.0)
        prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, max_iter=500, tol=1e-10)
        x, r = A.solve(b, params=prm)
        x_ref, r_ref = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, max_iter=500,
                                    tol=1e-10)
        assert r["info"] == 1 and abs(r["iters"] - r_ref["iters"]) <= 1
        assert rel(x, x_ref) < 1e-8
    finally:
        ctx.set_wait_limit(0.0)
        A.free()


def test_abort_word_cancels_a_running_solve(ctx):
    """A solve that would run for many seconds (tolerance 1e-300, 10^6 iterations) is cancelled
    from another host thread; it returns EGPU_ERR_ABORT promptly, and after the word is cleared
    the same matrix solves correctly."""
    import oracle

    m = meshgen.hex_cube(64)
    p, _, _, v, b, _ = poisson_problem(m, sym=True)
    A = eg.Matrix(ctx, eg.CRSPattern(p.n, p.nnz, 1, p.perm, p.rows, p.cols, p.diag), v)
    out = {}

    def run():
        t0 = time.perf_counter()
        try:
            A.solve(b, params=eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, max_iter=1000000, tol=1e-300,
                                              abort_not_converged=False))
            out["rc"] = "returned"
        except _lib.LibError as e:
            out["rc"] = e.code
        out["t"] = time.perf_counter() - t0

    try:
        th = threading.Thread(target=run)
        th.start()
        time.sleep(0.5)
        t_abort = time.perf_counter()
        ctx.abort(True)
        th.join(timeout=60)
        assert not th.is_alive()
        assert out["rc"] == -7, out  # EGPU_ERR_ABORT
        assert time.perf_counter() - t_abort < 2.0
        # still raised: the next call is refused too
        with pytest.raises(_lib.LibError) as ei:
            A.solve(b, params=eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, max_iter=100, tol=1e-10))
        assert ei.value.code == -7
        ctx.abort(False)
        prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, max_iter=5000, tol=1e-10)
        x, r = A.solve(b, params=prm)
        x_ref, r_ref = oracle.solve(p, v, b, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=5000,
                                    tol=1e-10)
        assert r["info"] == 1 and abs(r["iters"] - r_ref["iters"]) <= 1
        assert rel(x, x_ref) < 1e-8
    finally:
        ctx.abort(False)
        A.free()
