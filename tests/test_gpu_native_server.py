"""The library's native solve server (egpu_server_*, worker thread in C++) on short request
streams (needs a B200).

Every request solved inside the server's changing batch must equal the same system solved
alone by the FP64 drop-in path (or the oracle) within 1e-8 relative.
"""
import time

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen, server
from helpers import poisson_problem, rel

pytestmark = pytest.mark.gpu


def _pat(p):
    return eg.CRSPattern(p.n, p.nnz, p.dofs, p.perm, p.rows, p.cols, p.diag)


@pytest.mark.parametrize("method,prec", [(eg.BICGSTAB, eg.PREC_ILU0), (eg.CG, eg.PREC_DIAGONAL)])
def test_native_server_host_values(method, prec):
    """Values and RHS from the host: five systems on one registered pattern."""
    prm = eg.SolverParams(method=method, precond=prec, tol=1e-12, max_iter=5000, inner_tol=3e-4)
    mesh = meshgen.hex_cube(8)
    systems = []
    for s in range(5):
        k = meshgen.lognormal_conductivity(mesh.nelem, 0.5, 10 + s)
        p, _, _, v, b, _ = poisson_problem(mesh, elem_k=k, load=np.full(mesh.nnodes, 1.0 + s), sym=True)
        systems.append((p, v, b))
    srv = server.NativeSolveServer(0, prm, hbm_budget=1e9, chunk=8, max_resident=3)
    try:
        pid = srv.pattern(_pat(systems[0][0]))
        ids = [srv.submit(pid, v, b) for _, v, b in systems]
        for (p, v, b), rid in zip(systems, ids):
            x, res = srv.wait(rid, p.n, timeout=120.0)
            assert res["info"] == 1 and res["refinements"] >= 1
            assert res["seconds"] >= res["seconds_setup"] >= 0.0
            x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=prec, max_iter=5000, tol=1e-12)
            assert r_ref["info"] == 1
            assert rel(x, x_ref) < 1e-8
        info = srv.info()
        assert info["done"] == 5 and info["resident"] == 0 and info["queued"] == 0 and info["steps"] >= 1
        assert info["used_bytes"] == pytest.approx(0.0, abs=1.0)
        # transfers: every request's Values and RHS up, its solution down; the batch launched kernels
        n, nnz = systems[0][0].n, systems[0][0].nnz
        assert info["bytes_h2d"] == 5 * 8 * (nnz + n) and info["bytes_d2h"] == 5 * 8 * n
        assert info["kernel_launches"] >= info["steps"]
        with pytest.raises(Exception):
            srv.poll(ids[0])  # released by wait
    finally:
        srv.close()


def test_native_server_stream_equals_alone(ctx):
    """Device-assembled Poisson requests arriving over time, against the FP64 path alone."""
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=1e-12, max_iter=5000, inner_tol=3e-4,
                          abort_not_converged=False)
    reqs = server.poisson_stream(12, rate=500.0, m_lo=4, m_hi=14, seed=7)
    srv = server.NativeSolveServer(0, prm, hbm_budget=64e6, chunk=8, max_resident=4)
    try:
        stats = srv.run(reqs, keep_solutions=True)
    finally:
        srv.close()
    assert stats["solves"] == 12 and stats["converged"] == 12
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    assert stats["kernel_launches"] > 0 and stats["bytes_h2d"] > 0
    assert stats["bytes_d2h"] == 8 * sum((r.m + 1) ** 3 for r in reqs)  # one solution of n = (m+1)^3 each
    protos = {m: server.MeshPrototype(ctx, m, eg.PREC_ILU0) for m in sorted({r.m for r in reqs})}
    alone = [server.Request(r.rid, r.m, r.seed, 0.0) for r in reqs]
    server.run_one_at_a_time(ctx, eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=1e-12,
                                                  max_iter=5000), alone, protos, keep_solutions=True)
    for r, a in zip(reqs, alone):
        assert a.result["info"] == 1
        assert rel(r.x, a.x) < 1e-8, r.rid


def test_native_server_budget_runs_one_at_a_time():
    """A budget below one system's footprint still serves every request, one at a time."""
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=1e-10, max_iter=5000)
    srv = server.NativeSolveServer(0, prm, hbm_budget=1.0, chunk=4, max_resident=8)
    try:
        pid = srv.mesh_prototype(6)
        mesh, pat, con = srv.patterns[6][1]
        ids = [srv.submit_poisson(pid, load=np.full(mesh.nnodes, 1.0 + i), con=con) for i in range(4)]
        peak = 0
        results = {}
        while len(results) < len(ids):
            peak = max(peak, srv.info()["resident"])
            for rid in ids:
                if rid not in results:
                    got = srv.poll(rid, pat.n)
                    if got is not None:
                        results[rid] = got
            time.sleep(0.001)
        assert peak <= 1
        xs = [results[rid][0] for rid in ids]
        for i, x in enumerate(xs):  # load (1 + i) scales the solution linearly
            assert results[ids[i]][1]["info"] == 1
            assert rel(x, (1.0 + i) * xs[0]) < 1e-8
    finally:
        srv.close()
