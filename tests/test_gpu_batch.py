"""Batched mixed-precision solver (egpu_batch_*) against the oracle and against itself alone (needs a B200).

Every system is solved to tol on ||A x - b|| / ||b|| of its scaled system; the check is
the solution within 1e-8 relative of the oracle's FP64 solution at the same tolerance,
and the same system solved alone and inside a mix of others within 1e-8.
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


def _tet_system(m, seed):
    mesh = meshgen.tet_cube(m)
    k = meshgen.lognormal_conductivity(mesh.nelem, 0.5, seed)
    rng = np.random.default_rng(seed)
    p, _, _, v, _, con = poisson_problem(mesh, elem_k=k, sym=True)
    b = rng.random(p.n)
    b[con - 1] = 0.0
    return p, v, b


def _hex_system(m, seed):
    mesh = meshgen.hex_cube(m)
    k = meshgen.lognormal_conductivity(mesh.nelem, 1.0, seed)
    p, _, _, v, b, _ = poisson_problem(mesh, elem_k=k, load=meshgen.sine_source(mesh.coords))
    return p, v, b


TOL = 1e-11


@pytest.mark.parametrize("method,prec,make,sizes", [
    (eg.CG, eg.PREC_DIAGONAL, _tet_system, [4, 9, 6, 12, 5, 7]),
    (eg.CG, eg.PREC_NONE, _tet_system, [5, 8]),
    (eg.BICGSTAB, eg.PREC_ILU0, _hex_system, [6, 10, 8, 5]),
    (eg.BICGSTAB, eg.PREC_DIAGONAL, _hex_system, [7, 5, 9]),
])
def test_batch_matches_oracle(ctx, method, prec, make, sizes):
    systems = [make(m, 10 + i) for i, m in enumerate(sizes)]
    prm = eg.SolverParams(method=method, precond=prec, tol=TOL, max_iter=5000, inner_tol=3e-4)
    B = eg.Batch(ctx, prm, chunk=16)
    ids = [B.add(_pat(p), v, b) for p, v, b in systems]
    B.solve()
    for sid, (p, v, b) in zip(ids, systems):
        r = B.result(sid)
        assert r["info"] == 1, r
        x_ref, r_ref = oracle.solve(p, v, b, method=method, precond=prec, max_iter=5000, tol=TOL)
        assert rel(B.solution(sid), x_ref) < 1e-8
    B.free()


def test_same_alone_and_in_the_mix(ctx):
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=1e-12, max_iter=5000, inner_tol=3e-4)
    target = _hex_system(9, 3)
    others = [_hex_system(m, 20 + m) for m in (5, 12, 7, 11)]
    alone = eg.Batch(ctx, prm)
    sid = alone.add(_pat(target[0]), target[1], target[2])
    alone.solve()
    x_alone = alone.solution(sid)
    alone.free()
    mix = eg.Batch(ctx, prm, chunk=8)
    for p, v, b in others[:2]:
        mix.add(_pat(p), v, b)
    sid2 = mix.add(_pat(target[0]), target[1], target[2])
    for p, v, b in others[2:]:
        mix.add(_pat(p), v, b)
    mix.solve()
    assert rel(mix.solution(sid2), x_alone) < 1e-8
    mix.free()


def test_admission_while_running(ctx):
    """Systems added while others are mid-solve (continuous batching) finish with the right answer."""
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=TOL, max_iter=5000, inner_tol=3e-4)
    B = eg.Batch(ctx, prm, chunk=4)
    first = [_tet_system(m, 40 + m) for m in (10, 8)]
    later = [_tet_system(m, 60 + m) for m in (6, 9, 5)]
    ids = {B.add(_pat(p), v, b): (p, v, b) for p, v, b in first}
    finished = set()
    for _ in range(3):
        finished.update(B.step())
    assert B.pending() > 0
    for p, v, b in later:
        ids[B.add(_pat(p), v, b)] = (p, v, b)
    guard = 0
    while B.pending() > 0:
        finished.update(B.step())
        guard += 1
        assert guard < 100000
    assert finished == set(ids)
    for sid, (p, v, b) in ids.items():
        x_ref, _ = oracle.solve(p, v, b, method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=5000, tol=TOL)
        assert rel(B.solution(sid), x_ref) < 1e-8
    # freed slots are reused
    victim = next(iter(ids))
    B.remove(victim)
    p, v, b = later[0]
    assert B.add(_pat(p), v, b) == victim
    B.free()


@pytest.mark.parametrize("method,prec,make", [(eg.CG, eg.PREC_DIAGONAL, _tet_system),
                                              (eg.BICGSTAB, eg.PREC_ILU0, _hex_system)])
def test_autotuner_keeps_results_and_reports_every_system(ctx, method, prec, make):
    """egpu_batch_tune runs real steps: afterwards every system is still solved to the oracle's
    answer, and each one is listed as finished exactly once by the step loop."""
    sizes = [3, 4, 5, 6, 7, 8, 9, 10, 4, 6, 8, 5]
    systems = [make(m, 40 + i) for i, m in enumerate(sizes)]
    prm = eg.SolverParams(method=method, precond=prec, tol=TOL, max_iter=5000, inner_tol=3e-4)
    B = eg.Batch(ctx, prm, chunk=16)
    ids = [B.add(_pat(p), v, b) for p, v, b in systems]
    cfg = B.tune()
    assert cfg["candidates"] >= 1 and cfg["rate"] > 0
    assert cfg["chunk_iters"] in (16, 32, 64) and cfg["blocks_per_sm"] in (1, 2) and cfg["tri_mult"] in (1, 2, 4)
    assert cfg["slices_per_warp"] in (1, 2)  # rows per warp in the SpMV phases: 32 or 64
    seen = []
    for _ in range(100000):
        seen += B.step()
        if B.pending() == 0:
            seen += B.step()  # lists any system that finished in the last step's refinement check
            break
    assert sorted(seen) == sorted(ids)
    for sid, (p, v, b) in zip(ids, systems):
        assert B.result(sid)["info"] == 1
        x_ref, _ = oracle.solve(p, v, b, method=method, precond=prec, max_iter=5000, tol=TOL)
        assert rel(B.solution(sid), x_ref) < 1e-8
    B2 = eg.Batch(ctx, prm)
    B2.set_config(cfg)
    B2.free()
    B.free()
