"""Continuous-batching server (elmerfem_b200.server) on a short request stream (needs a B200).

Each request's result from the server (solved inside a changing mix of resident systems)
must equal the same request solved alone by the FP64 drop-in path within 1e-8 relative.
"""
import numpy as np
import pytest

import elmerfem_b200 as eg
from elmerfem_b200 import server

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("method,prec", [(eg.BICGSTAB, eg.PREC_ILU0), (eg.CG, eg.PREC_DIAGONAL)])
def test_server_results_equal_alone(ctx, method, prec):
    prm = eg.SolverParams(method=method, precond=prec, tol=1e-12, max_iter=5000, inner_tol=3e-4,
                          abort_not_converged=False)
    reqs = server.poisson_stream(10, rate=2000.0, m_lo=4, m_hi=12, seed=5)
    srv = server.SolveServer(ctx, prm, hbm_budget=64e6, chunk=8, max_resident=4)
    stats = srv.run(reqs, keep_solutions=True)
    assert stats["solves"] == 10 and stats["converged"] == 10
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    alone = [server.Request(r.rid, r.m, r.seed, 0.0) for r in reqs]
    server.run_one_at_a_time(ctx, eg.SolverParams(method=method, precond=prec, tol=1e-12, max_iter=5000),
                             alone, srv.protos, keep_solutions=True)
    for r, a in zip(reqs, alone):
        assert a.result["info"] == 1
        assert _rel(r.x, a.x) < 1e-8, r.rid


def test_admission_respects_budget(ctx):
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=1e-10, max_iter=5000)
    reqs = server.poisson_stream(6, rate=1e6, m_lo=10, m_hi=10, seed=9)
    srv = server.SolveServer(ctx, prm, chunk=4)
    one = srv.footprint(reqs[0])
    srv.budget = 2.5 * one  # two resident systems at most
    seen = []
    orig = srv._admit

    def spy(req, now):
        orig(req, now)
        seen.append(len(srv.resident))

    srv._admit = spy
    stats = srv.run(reqs)
    assert stats["solves"] == 6 and max(seen) <= 2
