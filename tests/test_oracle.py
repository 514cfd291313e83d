"""The oracle against the reference's own regression targets and internal invariants (CPU)."""
import json
import os

import numpy as np
import pytest

import oracle
from elmerfem_b200 import meshgen
from helpers import poisson_problem

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _heateq():
    d = np.load(os.path.join(GOLDEN, "heateq_mesh.npz"))
    return meshgen.Mesh(d["coords"], 303, d["elements"], 202, d["bnd_elements"], d["bnd_ids"], ())


def test_golden_targets_present():
    t = json.load(open(os.path.join(GOLDEN, "targets.json")))
    assert t["heateq"]["nrm"] == pytest.approx(0.0768016492512, rel=1e-12)


@pytest.mark.parametrize("method,prec", [(oracle.BICGSTAB, oracle.PREC_ILU0), (oracle.CG, oracle.PREC_ILU0),
                                         (oracle.CG, oracle.PREC_DIAGONAL), (oracle.BICGSTAB, oracle.PREC_NONE)])
@pytest.mark.parametrize("sym", [False, True])
def test_heateq_nrm(method, prec, sym):
    """fem/tests/heateq/TempDist.sif: k=1, source 1, T=0 on all boundaries, NRM=0.768016492512E-01
    (findnorm EPS 1e-5; the restatement reproduces it to ~1e-11)."""
    t = json.load(open(os.path.join(GOLDEN, "targets.json")))["heateq"]
    m = _heateq()
    p, _, _, v, b, _ = poisson_problem(m, sym=sym)
    x, r = oracle.solve(p, v, b, method=method, precond=prec, max_iter=350, tol=1e-12)
    assert r["info"] == 1
    nrm = oracle.compute_norm(x)
    assert abs(nrm - t["nrm"]) / t["nrm"] < 1e-9


@pytest.mark.parametrize("case,method", [(5, oracle.CG), (10, oracle.BICGSTAB)])
def test_linearsolvers_nrm(case, method):
    """fem/tests/linearsolvers/TempDist.sif: no source, T=case on all boundaries, ILU0, tol 1e-12 => NRM=case."""
    m = _heateq()
    p = oracle.create_pattern(m)
    vals, _ = oracle.assemble_poisson(m, p, nodal_k=np.ones(m.nnodes), load=None)
    con = np.sort(p.perm[m.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)
    b = np.zeros(p.n)
    oracle.dirichlet(p, vals, b, con, con_vals=np.full(con.size, float(case)))
    x, r = oracle.solve(p, vals, b, method=method, precond=oracle.PREC_ILU0, max_iter=3500, tol=1e-12)
    assert r["info"] == 1
    assert abs(oracle.compute_norm(x) - case) / case < 1e-9


def test_bandwidth_optimisation_accepted_on_heateq():
    m = _heateq()
    p = oracle.create_pattern(m)
    assert p.rejected == 0 and p.hbw_after < p.hbw_before
    assert sorted(p.perm.tolist()) == list(range(1, m.nnodes + 1))


def test_bandwidth_optimisation_rejected_on_structured_cube():
    p = oracle.create_pattern(meshgen.hex_cube(6))
    assert p.rejected == 1 and np.array_equal(p.perm, np.arange(1, 7 ** 3 + 1))


def test_ilu0_lusolve_inverts_tridiagonal_exactly():
    """ILU0 of a tridiagonal matrix is its exact LU (no fill), so LU-solve inverts it."""
    n = 50
    rows = np.arange(1, 3 * n, 3, dtype=np.int32)
    rows = np.concatenate([[1], np.cumsum([2] + [3] * (n - 2) + [2]) + 1]).astype(np.int32)
    cols, vals, diag = [], [], []
    for i in range(n):
        for j in (i - 1, i, i + 1):
            if 0 <= j < n:
                if j == i:
                    diag.append(len(cols) + 1)
                cols.append(j + 1)
                vals.append(4.0 if i == j else -1.0)
    pat = oracle.Pattern(n, len(cols), 1, np.arange(1, n + 1, dtype=np.int32), rows, np.array(cols, np.int32),
                         np.array(diag, np.int32), 0, 0, 0, 0)
    vals = np.array(vals)
    ilu = oracle.ilu0(pat, vals)
    rhs = np.random.default_rng(0).random(n)
    x = oracle.lusolve(pat, ilu, rhs)
    assert np.allclose(oracle.spmv(pat, vals, x), rhs, rtol=0, atol=1e-13)


def test_hex_stiffness_row_sums_vanish():
    """Constant fields are in the kernel of the Laplacian: interior row sums are ~0."""
    m = meshgen.hex_cube(4)
    p = oracle.create_pattern(m)
    vals, _ = oracle.assemble_poisson(m, p, nodal_k=np.ones(m.nnodes), load=None)
    s = oracle.spmv(p, vals, np.ones(p.n))
    assert np.max(np.abs(s)) < 1e-13


def test_zero_rhs_short_cut():
    m = meshgen.hex_cube(3)
    p, _, _, v, _, _ = poisson_problem(m)
    x, r = oracle.solve(p, v, np.zeros(p.n), method=oracle.CG, precond=oracle.PREC_DIAGONAL, max_iter=10)
    assert r["info"] == 1 and not np.any(x)


@pytest.mark.parametrize("mk", [lambda: meshgen.hex_cube(4), lambda: meshgen.tet_cube(4)], ids=["hex", "tet"])
def test_poisson_patch_and_load_integral(mk):
    """Pins the restated diffusion compose by properties of the exact Galerkin matrix: a linear
    field is reproduced exactly by trilinear hexes and linear tets (the patch test: K u = 0 at
    every interior node, for k constant), the energy u^T K u of u = x equals k * volume, and a
    unit load integrates to the volume (sum of the load vector = 1 on the unit cube)."""
    m = mk()
    p = oracle.create_pattern(m)
    k = 2.5
    vals, rhs = oracle.assemble_poisson(m, p, nodal_k=np.full(m.nnodes, k), load=np.ones(m.nnodes))
    xyz = m.coords
    row_of = p.perm - 1  # node -> row
    bnd = set((m.boundary_nodes(range(1, 7)) - 1).tolist())
    interior_rows = np.array([row_of[a] for a in range(m.nnodes) if a not in bnd])
    for c in range(3):
        u = np.zeros(p.n)
        u[row_of] = 0.3 + 1.7 * xyz[:, c]
        Ku = oracle.spmv(p, vals, u)
        assert np.max(np.abs(Ku[interior_rows])) < 1e-12
        ux = np.zeros(p.n)
        ux[row_of] = xyz[:, c]
        assert abs(ux @ oracle.spmv(p, vals, ux) - k * 1.0) < 1e-12
    assert abs(rhs.sum() - 1.0) < 1e-13


@pytest.mark.parametrize("mk", [lambda: meshgen.hex_cube(3), lambda: meshgen.tet_cube(3)], ids=["hex", "tet"])
def test_elastic_rigid_body_modes_and_load(mk):
    """Pins the restated StressCompose: the three translations and three infinitesimal
    rotations of the body are strain-free, so K u = 0 in every row; a uniform stretch
    u = e x along x has energy u^T K u = C11 e^2 * volume with C11 = E(1-nu)/((1+nu)(1-2nu));
    and a body force b integrates to b * volume per component."""
    m = mk()
    p = oracle.create_pattern(m, dofs=3)
    E, nu, bf = 200e9, 0.3, (1.0, -2.0, 3.0)
    vals, rhs = oracle.assemble_elastic(m, p, E, nu, bf)
    xyz = m.coords
    base = (p.perm - 1) * 3
    scale = np.abs(vals).max()
    modes = []
    for d in range(3):
        u = np.zeros(p.n)
        u[base + d] = 1.0
        modes.append(u)
    for (i, j) in ((0, 1), (1, 2), (2, 0)):
        u = np.zeros(p.n)
        u[base + i] = -xyz[:, j]
        u[base + j] = xyz[:, i]
        modes.append(u)
    for u in modes:
        assert np.max(np.abs(oracle.spmv(p, vals, u))) < 1e-12 * scale
    e = 1e-3
    u = np.zeros(p.n)
    u[base] = e * xyz[:, 0]
    c11 = E * (1 - nu) / ((1 + nu) * (1 - 2 * nu))
    assert abs(u @ oracle.spmv(p, vals, u) / (c11 * e * e) - 1.0) < 1e-12
    for d in range(3):
        assert abs(rhs[np.arange(p.n) % 3 == d].sum() - bf[d]) < 1e-12 * abs(bf[d])


def test_dirichlet_variants_agree_and_reproduce_linear_fields():
    """Pins the restated DefaultDirichletBCs: with the boundary values of a linear field and no
    load, both variants (row replacement, symmetric elimination) give the linear field itself
    (the discrete solution is exact for it); the symmetric variant leaves a symmetric matrix."""
    m = meshgen.hex_cube(5)
    p = oracle.create_pattern(m)
    vals, rhs = oracle.assemble_poisson(m, p, nodal_k=np.ones(m.nnodes), load=None)
    nodes = m.boundary_nodes(range(1, 7)) - 1
    con = (p.perm[nodes]).astype(np.int32)  # 1-based rows
    order = np.argsort(con)
    con, nodes = con[order], nodes[order]
    field = 1.0 + 2.0 * m.coords[:, 0] - 0.5 * m.coords[:, 1] + 0.25 * m.coords[:, 2]
    exact = np.zeros(p.n)
    exact[p.perm - 1] = field
    for sym in (False, True):
        v, b = vals.copy(), rhs.copy()
        oracle.dirichlet(p, v, b, con, field[nodes], symmetric=sym)
        x, r = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, max_iter=500, tol=1e-12)
        assert r["info"] == 1
        assert np.max(np.abs(x - exact)) < 1e-9
        if sym:
            A = np.zeros((p.n, p.n))
            for i in range(p.n):
                for kk in range(p.rows[i] - 1, p.rows[i + 1] - 1):
                    A[i, p.cols[kk] - 1] = v[kk]
            assert np.max(np.abs(A - A.T)) < 1e-14 * np.abs(A).max()
