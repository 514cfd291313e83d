"""Team solver of egpu_batch_solve (CG with M = I or Jacobi).

Each system's whole mixed-precision solve (FP64 residual, FP32 inner CG segments with reliable
updating, FP64 update) runs on a team of CTAs of one launch: one CTA for a small system, several
for a large one, which split its slices and meet at a barrier of their own.  Every solution must
meet 1e-8 against the oracle's FP64 solve at the same tolerance, as on the stepwise path
(EGPU_BATCH_TEAMS=0), whose results it must also match.
"""
import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen
from helpers import poisson_problem, rel

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


def _tet_system(m, seed, zero_rhs=False):
    mesh = meshgen.tet_cube(m)
    k = meshgen.lognormal_conductivity(mesh.nelem, 0.5, seed)
    rng = np.random.default_rng(seed)
    p, _, _, v, _, con = poisson_problem(mesh, elem_k=k, sym=True)
    b = np.zeros(p.n) if zero_rhs else rng.random(p.n)
    b[con - 1] = 0.0
    return p, v, b


def _run(ctx, monkeypatch, systems, teams, **kw):
    monkeypatch.setenv("EGPU_BATCH_TEAMS", "1" if teams else "0")
    prm = eg.SolverParams(method=eg.CG, precond=kw.pop("precond", eg.PREC_DIAGONAL), tol=TOL,
                          max_iter=kw.pop("max_iter", 5000), inner_tol=3e-4, **kw)
    B = eg.Batch(ctx, prm, chunk=16)
    try:
        ids = [B.add(_pat(p), v, b) for p, v, b in systems]
        B.solve()
        return [B.result(i) for i in ids], [B.solution(i) for i in ids]
    finally:
        B.free()


# sizes 24 and 30 (15,625 and 29,791 rows) get teams of several CTAs next to one-CTA teams
@pytest.mark.parametrize("prec,oprec", [(eg.PREC_DIAGONAL, oracle.PREC_DIAGONAL), (eg.PREC_NONE, oracle.PREC_NONE)])
def test_teams_match_oracle_and_stepwise_path(ctx, monkeypatch, prec, oprec):
    systems = [_tet_system(m, 20 + i) for i, m in enumerate([4, 9, 24, 30, 6, 12, 3])]
    res_t, xs_t = _run(ctx, monkeypatch, systems, True, precond=prec)
    res_s, xs_s = _run(ctx, monkeypatch, systems, False, precond=prec)
    it_t = it_s = 0
    for (p, v, b), rt, xt, rs, xs in zip(systems, res_t, xs_t, res_s, xs_s):
        x_ref, _ = oracle.solve(p, v, b, method=oracle.CG, precond=oprec, max_iter=5000, tol=TOL)
        assert rt["info"] == 1 and rt["residual"] < TOL, rt
        assert rel(xt, x_ref) < 1e-8 and rel(xs, x_ref) < 1e-8
        it_t += rt["iters"]
        it_s += rs["iters"]
    # the two paths run the same refinement with two forms of the inner CG (three-phase on the
    # teams, single-reduction on the stepwise kernel): about the same work
    assert abs(it_t - it_s) <= 0.15 * it_s, (it_t, it_s)


def test_zero_rhs_unscaled_jacobi_and_iteration_limit(ctx, monkeypatch):
    systems = [_tet_system(10, 31), _tet_system(8, 32, zero_rhs=True), _tet_system(26, 33)]
    # a zero right-hand side is answered at admission (x = 0); without scaling the diagonal is not
    # one, so Jacobi divides by it
    res, xs = _run(ctx, monkeypatch, systems, True, scale_system=False)
    for (p, v, b), r, x in zip(systems, res, xs):
        assert r["info"] == 1, r
        if not b.any():
            assert not np.asarray(x).any()
            continue
        x_ref, _ = oracle.solve(p, v, b, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=5000, tol=TOL,
                                scale=False)
        assert rel(x, x_ref) < 1e-8
    # the iteration limit ends every solve with HUTI_MAXITER, as on the stepwise path
    res_t, _ = _run(ctx, monkeypatch, systems, True, max_iter=20)
    res_s, _ = _run(ctx, monkeypatch, systems, False, max_iter=20)
    for (p, v, b), rt, rs in zip(systems, res_t, res_s):
        want = 1 if not b.any() else 2
        assert rt["info"] == want and rs["info"] == want, (rt, rs)


def test_many_systems_every_result_reported(ctx, monkeypatch):
    """More systems than CTAs: each CTA takes tasks from the queue until it is empty."""
    rng = np.random.default_rng(7)
    sizes = [int(v) for v in rng.integers(2, 9, size=300)] + [22, 28]
    systems = [_tet_system(m, 100 + i) for i, m in enumerate(sizes)]
    res, xs = _run(ctx, monkeypatch, systems, True)
    for j in list(range(0, len(systems), 37)) + [len(systems) - 2, len(systems) - 1]:
        p, v, b = systems[j]
        x_ref, _ = oracle.solve(p, v, b, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=5000, tol=TOL)
        assert rel(xs[j], x_ref) < 1e-8, j
    assert all(r["info"] == 1 for r in res)


def test_abort_word_cancels_the_team_solver(ctx, monkeypatch):
    """A batched solve that would run for seconds (tolerance 1e-300; it ends by itself at 200,000
    inner iterations a system) is cancelled from another host thread: it returns EGPU_ERR_ABORT
    promptly, and once the word is cleared the context solves a batch as the oracle does."""
    import threading
    import time

    from elmerfem_b200 import _lib

    monkeypatch.setenv("EGPU_BATCH_TEAMS", "1")
    systems = [_tet_system(m, 60 + i) for i, m in enumerate([20, 24, 6, 9])]
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=1e-300, max_iter=200000,
                          max_refinements=1000000, inner_tol=3e-4)
    B = eg.Batch(ctx, prm)
    out = {}

    def run():
        try:
            B.solve()
            out["rc"] = "returned"
        except _lib.LibError as e:
            out["rc"] = e.code

    try:
        for p, v, b in systems:
            B.add(_pat(p), v, b)
        th = threading.Thread(target=run)
        th.start()
        time.sleep(0.3)
        t_abort = time.perf_counter()
        ctx.abort(True)
        th.join(timeout=60)
        assert not th.is_alive()
        assert out["rc"] == -7, out  # EGPU_ERR_ABORT
        assert time.perf_counter() - t_abort < 2.0
    finally:
        ctx.abort(False)
        B.free()
    res, xs = _run(ctx, monkeypatch, systems, True)
    for (p, v, b), r, x in zip(systems, res, xs):
        x_ref, _ = oracle.solve(p, v, b, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=5000, tol=TOL)
        assert r["info"] == 1 and rel(x, x_ref) < 1e-8
