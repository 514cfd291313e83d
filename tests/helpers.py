"""Problem set-up shared by the tests: the same mesh fed to the oracle and to the GPU."""
import numpy as np

import oracle
from elmerfem_b200 import meshgen


def poisson_problem(mesh, elem_k=None, load=None, sym=False, bc_ids=range(1, 7)):
    """Oracle-assembled Poisson system with zero Dirichlet on bc_ids."""
    p = oracle.create_pattern(mesh)
    if load is None:
        load = np.ones(mesh.nnodes)
    nodal_k = None if elem_k is not None else np.ones(mesh.nnodes)
    vals, rhs = oracle.assemble_poisson(mesh, p, elem_k=elem_k, nodal_k=nodal_k, load=load)
    con = np.sort(p.perm[mesh.boundary_nodes(bc_ids) - 1]).astype(np.int32)
    v, b = vals.copy(), rhs.copy()
    oracle.dirichlet(p, v, b, con, symmetric=sym)
    return p, vals, rhs, v, b, con


def elastic_problem(mesh, E=200e9, nu=0.3, bf=(0.0, 0.0, -1e4)):
    p = oracle.create_pattern(mesh, dofs=3)
    vals, rhs = oracle.assemble_elastic(mesh, p, E, nu, bf)
    nodes = mesh.boundary_nodes([1])
    con = np.sort(np.concatenate([3 * (p.perm[nodes - 1] - 1) + d for d in (1, 2, 3)])).astype(np.int32)
    v, b = vals.copy(), rhs.copy()
    oracle.dirichlet(p, v, b, con, symmetric=False)
    return p, vals, rhs, v, b, con


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def row_rel_max(pat, a, b):
    """max over entries |a-b| / max|row of b| (relative to the row's scale)"""
    a, b = np.asarray(a), np.asarray(b)
    rows = pat.rows - 1
    scale = np.maximum.reduceat(np.abs(b), rows[:-1])
    per = np.repeat(scale, np.diff(rows))
    return float(np.max(np.abs(a - b) / np.maximum(per, 1e-300)))


def renumbered(mesh, seed):
    """The same mesh with its nodes numbered in a random order (boundary elements follow)."""
    from elmerfem_b200 import meshgen

    rng = np.random.default_rng(seed)
    new = rng.permutation(mesh.nnodes)  # old node -> new node (0-based)
    coords = np.empty_like(mesh.coords)
    coords[new] = mesh.coords
    return meshgen.Mesh(coords, mesh.elem_code, (new[mesh.elements - 1] + 1).astype(np.int32), mesh.bnd_code,
                        (new[mesh.bnd_elements - 1] + 1).astype(np.int32), mesh.bnd_ids)
