"""The oracle's GCR and BiCGStab(l) restatements, pinned on the CPU.

The reference's tests give only NRM targets for these methods' solutions, so the oracle's
restatements (fem/src/IterativeMethods.src: GCR :919-1055, BiCGStab(l) :559-834) are pinned
here by an independent numpy transcription of GCR (same iterates up to the order of the dot
product sums: iteration counts within one, solutions within 1e-12), by GCR's defining
property (without restarts the residual never grows: each step minimises it over the new
direction), and by BiCGStab(l) solving a Poisson system to the requested tolerance in about
as many BiCG steps as BiCGStab takes.
"""
import numpy as np
import pytest

import oracle
from elmerfem_b200 import meshgen


def _system(seed=1, m=4):
    p = oracle.create_pattern(meshgen.hex_cube(m))
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1.0, 1.0, p.nnz)
    v[p.diag - 1] = np.diff(p.rows) + 2.0
    b = rng.uniform(-1.0, 1.0, p.n)
    return p, v, b


def _dense(p, v):
    A = np.zeros((p.n, p.n))
    for i in range(p.n):
        for k in range(p.rows[i] - 1, p.rows[i + 1] - 1):
            A[i, p.cols[k] - 1] = v[k]
    return A


def _numpy_gcr(A, b, m, tol, maxit, diag_prec):
    """GCR with restart m (IterativeMethods.src:919-1055), x0 = 1e-8 as IterSolver sets it."""
    n = len(b)
    d = np.diag(A).copy()
    pc = (lambda r: np.where(np.abs(d) > 10 * 2.220446049250313e-16, r / d, r)) if diag_prec else (lambda r: r.copy())
    x = np.full(n, 1e-8)
    r = b - A @ x
    bnorm = np.linalg.norm(b)
    S, V = [None] * (m - 1), [None] * (m - 1)
    hist = [np.linalg.norm(r) / bnorm]
    for k in range(1, maxit + 1):
        if k % m == 0:
            j = m
        else:
            j = k % m
            if j == 1 and k > 1:
                r = b - A @ x
        T1 = pc(r)
        T2 = A @ T1
        for i in range(1, j):
            beta = V[i - 1] @ T2
            T1 = T1 - beta * S[i - 1]
            T2 = T2 - beta * V[i - 1]
        alpha = np.linalg.norm(T2)
        T1 = (1.0 / alpha) * T1
        T2 = (1.0 / alpha) * T2
        beta = T2 @ r
        x = x + beta * T1
        r = r - beta * T2
        if j != m:
            S[j - 1], V[j - 1] = T1, T2
        hist.append(np.linalg.norm(r) / bnorm)
        if hist[-1] < tol:
            return x, k, hist
    return x, maxit, hist


@pytest.mark.parametrize("restart", [3, 8, 200])
@pytest.mark.parametrize("prec", [oracle.PREC_NONE, oracle.PREC_DIAGONAL])
def test_gcr_matches_numpy_transcription(restart, prec):
    p, v, b = _system(seed=restart + prec)
    x_ref, r_ref = oracle.solve(p, v, b, method=oracle.GCR, precond=prec, max_iter=500, tol=1e-10, scale=False,
                                restart=restart)
    x_np, it_np, hist = _numpy_gcr(_dense(p, v), b, restart, 1e-10, 500, prec == oracle.PREC_DIAGONAL)
    assert r_ref["info"] == 1
    assert abs(r_ref["iters"] - it_np) <= 1, (r_ref["iters"], it_np)
    assert np.linalg.norm(x_ref - x_np) <= 1e-12 * np.linalg.norm(x_np) + 1e-14
    if restart >= it_np:  # no restart: the residual never grows
        assert all(h2 <= h1 * (1 + 1e-12) for h1, h2 in zip(hist, hist[1:]))


@pytest.mark.parametrize("degree,prec", [(2, oracle.PREC_NONE), (3, oracle.PREC_NONE), (4, oracle.PREC_NONE),
                                         (8, oracle.PREC_NONE), (2, oracle.PREC_DIAGONAL), (8, oracle.PREC_DIAGONAL),
                                         (2, oracle.PREC_ILU0), (3, oracle.PREC_ILU0), (4, oracle.PREC_ILU0)])
def test_bicgstabl_solves_to_tolerance(degree, prec):
    """On a 10^3 Poisson system with log-normal conductivity.  (A degree above the BiCG steps
    the solve needs can break down, as the reference's RealBiCGStabl does: not tested here.)"""
    from helpers import poisson_problem

    m = 10
    p, _, _, v, b, _ = poisson_problem(meshgen.hex_cube(m), elem_k=np.exp(np.random.default_rng(1).normal(0, 1, m ** 3)))
    A = _dense(p, v)
    x, r = oracle.solve(p, v, b, method=oracle.BICGSTABL, precond=prec, max_iter=500, tol=1e-10, restart=degree)
    assert r["info"] == 1
    assert np.linalg.norm(A @ x - b) <= 1e-8 * np.linalg.norm(b)
    x_exact = np.linalg.solve(A, b)
    assert np.linalg.norm(x - x_exact) <= 1e-6 * np.linalg.norm(x_exact)
    # a round of degree l takes l BiCG steps: about as many in all as BiCGStab's iterations
    _, r_b = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=prec, max_iter=500, tol=1e-10)
    assert r["iters"] * degree <= 1.5 * r_b["iters"] + degree
