"""The product's CreateMatrix (egpu_pattern_create, host C++) against the oracle: bit-exact Perm/Rows/Cols/Diag."""
import os

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import _lib, meshgen
from helpers import renumbered

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _heateq():
    d = np.load(os.path.join(GOLDEN, "heateq_mesh.npz"))
    return meshgen.Mesh(d["coords"], 303, d["elements"], 202, d["bnd_elements"], d["bnd_ids"], ())


@pytest.mark.parametrize("mesh", [lambda: meshgen.hex_cube(5), lambda: meshgen.hex_cube(3, 4, 7),
                                  lambda: meshgen.tet_cube(4), _heateq,
                                  lambda: renumbered(meshgen.hex_cube(4), 1), lambda: renumbered(meshgen.tet_cube(3), 2)],
                         ids=["hex5", "hex3x4x7", "tet4", "heateq", "hex4-shuffled", "tet3-shuffled"])
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


def _python_optimize_bandwidth(nn, lists, use_always=False):
    """OptimizeBandwidth (BandwidthOptimize.src:108-355) transcribed with the list pointers as
    (row, position) pairs: minimum-degree start, the depth-first Levelize with its explicit
    stack, the pseudo-peripheral search (with its `StartNode = j` assignment as written), the
    Cuthill-McKee numbering in list order from StartNode, reversed, and the rejection when the
    half bandwidth grows.  lists[i] (1-based nodes) are sorted and hold i itself."""
    deg = [0] + [len(lists[i]) for i in range(1, nn + 1)]

    def bandwidth(perm):
        return max(abs(perm[i] - perm[k]) for i in range(1, nn + 1) for k in lists[i])

    hb_before = bandwidth(list(range(nn + 1))) + 1
    level = [0] * (nn + 1)
    done = [False] * (nn + 1)
    state = {"max": 0}

    def levelize(nin, lev):
        n, L = nin, lev
        stack = []
        p = (n, 0) if lists[n] else None
        while p is not None:
            stack.append(p)
            level[n] = L
            done[n] = True
            state["max"] = max(state["max"], L)
            p = (n, 0) if lists[n] else None
            while True:
                if p is not None:
                    nn_ = lists[p[0]][p[1]]
                    if not done[nn_]:
                        n = nn_
                        L += 1
                        break
                elif stack:
                    p = stack.pop()
                    L -= 1
                else:
                    break
                p = (p[0], p[1] + 1) if p[1] + 1 < len(lists[p[0]]) else None

    start, mindeg = 1, deg[1]
    for i in range(1, nn + 1):
        if deg[i] < mindeg:
            start, mindeg = i, deg[i]
        level[i] = 0
    levelize(start, 0)
    newroot = True
    while newroot:
        newroot = False
        mindeg, k = deg[start], start
        for i in range(1, nn + 1):
            if level[i] == state["max"] and deg[i] < mindeg:
                k, mindeg = i, deg[i]
        if k != start:
            j = state["max"]
            state["max"] = 0
            for i in range(nn + 1):
                done[i] = False
            levelize(k, 0)
            if j > state["max"]:
                newroot = True
                start = j
    permlocal = [0] * (nn + 2)
    doneidx = [0] * (nn + 1)
    indx = 1
    permlocal[indx] = start
    doneidx[start] = indx
    indx += 1
    for i in range(1, nn + 1):
        if permlocal[i] == 0:
            for j in range(1, nn + 1):
                if doneidx[j] == 0:
                    permlocal[indx] = j
                    doneidx[j] = indx
                    indx += 1
                    break
        for k in lists[permlocal[i]]:
            if doneidx[k] == 0:
                permlocal[indx] = k
                doneidx[k] = indx
                indx += 1
    perm = [0] * (nn + 1)
    for i in range(1, nn + 1):
        perm[permlocal[i]] = nn - i + 1
    hb_after = bandwidth(perm) + 1
    rejected = hb_before < hb_after and not use_always
    if rejected:  # the routine then returns the original half bandwidth and ordering
        perm = list(range(nn + 1))
        hb_after = hb_before
    return perm[1:], hb_before, hb_after, start, rejected


@pytest.mark.parametrize("mk", [lambda: meshgen.hex_cube(4), lambda: meshgen.tet_cube(4), lambda: _heateq(),
                                lambda: renumbered(meshgen.hex_cube(4), 1), lambda: renumbered(meshgen.tet_cube(3), 2),
                                lambda: renumbered(_heateq(), 3)],
                         ids=["hex4", "tet4", "heateq", "hex4-shuffled", "tet3-shuffled", "heateq-shuffled"])
def test_bandwidth_optimisation_matches_transcription(mk):
    """The oracle's OptimizeBandwidth against a Python transcription of the reference's routine
    (structured meshes: rejected; shuffled node numbering and the heateq mesh: accepted)."""
    mesh = mk()
    nn = mesh.nnodes
    lists = [[] for _ in range(nn + 1)]
    adj = [set() for _ in range(nn + 1)]
    for el in mesh.elements:
        nodes = [int(q) for q in el]
        for a in nodes:
            adj[a].update(nodes)
    for a in range(1, nn + 1):
        lists[a] = sorted(adj[a])
    perm, hb, ha, start, rej = _python_optimize_bandwidth(nn, lists)
    p = oracle.create_pattern(mesh)
    assert (p.hbw_before, p.hbw_after, p.start_node, bool(p.rejected)) == (hb, ha, start, rej)
    assert np.array_equal(p.perm, np.array(perm, np.int32))
