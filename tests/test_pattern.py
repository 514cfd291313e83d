"""The product's CreateMatrix (egpu_pattern_create, host C++) against the oracle: bit-exact Perm/Rows/Cols/Diag."""
import os

import numpy as np
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen

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
