"""The product's CreateMatrix (egpu_pattern_create, host C++) against the oracle: bit-exact Perm/Rows/Cols/Diag."""
import os

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import _lib, meshgen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _heateq():
    d = np.load(os.path.join(GOLDEN, "heateq_mesh.npz"))
    return meshgen.Mesh(d["coords"], 303, d["elements"], 202, d["bnd_elements"], d["bnd_ids"], ())


@pytest.mark.parametrize("mesh", [lambda: meshgen.hex_cube(5), lambda: meshgen.hex_cube(3, 4, 7),
                                  lambda: meshgen.tet_cube(4), _heateq])
@pytest.mark.parametrize("dofs", [1, 3])
@pytest.mark.parametrize("opt", [True, False])
def test_pattern_bit_exact(mesh, dofs, opt):
    m = mesh()
    p = eg.create_matrix(m, dofs=dofs, optimize_bandwidth=opt)
    q = oracle.create_pattern(m, dofs=dofs, optimize=opt)
    assert (p.n, p.nnz) == (q.n, q.nnz)
    for a in ("perm", "rows", "cols", "diag"):
        assert np.array_equal(getattr(p, a), getattr(q, a)), a


def test_pattern_shuffled_element_order():
    """Element order does not change the sorted lists, hence not the pattern."""
    m = meshgen.tet_cube(3)
    m2 = meshgen.Mesh(m.coords, m.elem_code, m.elements[::-1].copy(), m.bnd_code, m.bnd_elements, m.bnd_ids)
    p, q = eg.create_matrix(m), eg.create_matrix(m2)
    assert np.array_equal(p.cols, q.cols) and np.array_equal(p.perm, q.perm)


def test_pattern_rejects_bad_connectivity():
    m = meshgen.hex_cube(2)
    bad = m.elements.copy()
    bad[0, 0] = m.nnodes + 5
    m2 = meshgen.Mesh(m.coords, 808, bad, 404, m.bnd_elements, m.bnd_ids)
    with pytest.raises(eg.LibError):
        eg.create_matrix(m2)


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("mk", [lambda: meshgen.hex_cube(7), lambda: meshgen.tet_cube(6),
                                lambda: meshgen.hex_cube(4), lambda: _heateq()],
                         ids=["hex7", "tet6", "hex4", "heateq"])
def test_ilu_structure_matches_oracle(mk, order):
    """egpu_ilu_pattern (the library's host ILU(n) structure) equals the oracle's restatement
    of InitializeILU1 applied n times, entry for entry."""
    import ctypes as C
    mesh = mk()
    p = oracle.create_pattern(mesh)
    ref = oracle.ilu_pattern(p, order)
    L = _lib.lib()
    nz = L.egpu_ilu_pattern(p.n, p.rows, p.cols, p.diag, order, 0, None, None, None)
    assert nz == ref[1].size
    r, c, d = np.zeros(p.n + 1, np.int32), np.zeros(nz, np.int32), np.zeros(p.n, np.int32)
    assert L.egpu_ilu_pattern(p.n, p.rows, p.cols, p.diag, order, nz, r.ctypes.data, c.ctypes.data,
                              d.ctypes.data) == nz
    assert np.array_equal(r, ref[0]) and np.array_equal(c, ref[1]) and np.array_equal(d, ref[2])
    # the structure contains the matrix pattern and grows with the order
    assert nz >= p.nnz


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("mk", [lambda: meshgen.hex_cube(5), lambda: meshgen.tet_cube(5), lambda: _heateq()],
                         ids=["hex5", "tet5", "heateq"])
def test_ilu_structure_is_the_symbolic_product(mk, order):
    """Pins the oracle's ILU(n) structure by an independent construction: one InitializeILU1
    step (CRSMatrix.src:2391-2497) adds to the pattern S every (i, j) reached through some
    k < i with s_ik in S and j in the strictly upper part of S's row k, i.e. S | tril(S) @ triu(S)
    as boolean sparse matrices; ILU(n) applies the step n times."""
    import scipy.sparse as sp

    mesh = mk()
    p = oracle.create_pattern(mesh)
    S = sp.csr_matrix((np.ones(p.nnz), p.cols - 1, p.rows - 1), shape=(p.n, p.n))
    for _ in range(order):
        L, U = sp.tril(S, -1, format="csr"), sp.triu(S, 1, format="csr")
        S = ((S + L @ U) != 0).astype(np.float64).tocsr()
    S.sort_indices()
    r, c, d = oracle.ilu_pattern(p, order)
    assert np.array_equal(r - 1, S.indptr) and np.array_equal(c - 1, S.indices)
    assert np.all(c[d - 1] - 1 == np.arange(p.n))


@pytest.mark.parametrize("mk,dofs", [(lambda: meshgen.hex_cube(4), 1), (lambda: meshgen.tet_cube(4), 1),
                                     (lambda: meshgen.hex_cube(3), 3), (lambda: _heateq(), 1)],
                         ids=["hex4", "tet4", "hex3x3", "heateq"])
def test_pattern_is_the_element_adjacency(mk, dofs):
    """Pins the oracle's CRS creation (MakeListMatrix, CRS_CreateMatrix, CRS_SortMatrix) by an
    independent construction: under its own Perm, row (Perm(a)-1)*DOFs+i holds the columns
    (Perm(b)-1)*DOFs+j of every node b sharing an element with node a (a itself included), all
    DOFs coupled, sorted ascending, Diag pointing at the row's own column; Perm is a
    permutation of the nodes, and the optimised bandwidth never exceeds the original one."""
    mesh = mk()
    p = oracle.create_pattern(mesh, dofs=dofs)
    nn = mesh.nnodes
    assert sorted(p.perm.tolist()) == list(range(1, nn + 1))
    assert p.hbw_after <= p.hbw_before
    adj = [set() for _ in range(nn)]
    for el in mesh.elements:
        nodes = [int(q) - 1 for q in el]
        for a in nodes:
            adj[a].update(nodes)
    rows, cols = [0], []
    order = np.argsort(p.perm)  # node of each row block
    for a in order:
        bl = sorted((int(p.perm[b]) - 1) for b in adj[a])
        for i in range(dofs):
            for bb in bl:
                cols.extend(bb * dofs + j for j in range(dofs))
            rows.append(len(cols))
    assert np.array_equal(p.rows - 1, np.array(rows)) and np.array_equal(p.cols - 1, np.array(cols))
    assert np.all(p.cols[p.diag - 1] - 1 == np.arange(p.n))
