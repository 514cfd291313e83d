"""Size-independent properties of assembled systems and solutions.

They hold at any mesh size, so they check the device path at the full workload sizes where the
oracle would take minutes: the Galerkin matrix of the diffusion operator annihilates constants
and integrates the energy of a linear field exactly, the elasticity matrix annihilates the six
rigid-body modes, a unit load integrates to the volume, and a solve meets its stopping test on
the scaled system (SolverUtils.src:6470-6640 scaling, huti_cg_D.F90 / huti_bicgstab_D.F90
true-residual test).  The CPU tests apply the same functions to the oracle's systems.
"""
import numpy as np
import scipy.sparse as sp


def csr(pat, vals):
    """scipy CSR of a 1-based Matrix_t pattern and its values."""
    return sp.csr_matrix((np.asarray(vals, np.float64), np.asarray(pat.cols, np.int64) - 1,
                          np.asarray(pat.rows, np.int64) - 1), shape=(pat.n, pat.n))


def row_sum_defect(pat, vals):
    """max over rows |sum_j a_ij| / sum_j |a_ij| (0 for a matrix that annihilates constants)."""
    S = csr(pat, vals)
    s = np.abs(S @ np.ones(pat.n))
    a = np.abs(S) @ np.ones(pat.n)
    return float(np.max(s / np.maximum(a, 1e-300)))


def symmetry_defect(pat, vals):
    """max |a_ij - a_ji| / max |a|."""
    S = csr(pat, vals)
    return float(abs(S - S.T).max() / abs(S).max())


def nodal_field(pat, values_by_node, dofs=1, component=0):
    """A vector in row order holding values_by_node at DOF `component` of every node."""
    u = np.zeros(pat.n)
    u[(np.asarray(pat.perm, np.int64) - 1) * dofs + component] = values_by_node
    return u


def linear_field_energy_defect(mesh, pat, vals, elem_k):
    """|u^T K u - sum_e k_e vol_e| / sum_e k_e vol_e for u = x, y, z in turn (|grad u| = 1);
    elements of a cube split into equal volumes (hex_cube, tet_cube), vol_e = 1 / nelem."""
    S = csr(pat, vals)
    target = float(np.sum(elem_k)) / mesh.nelem
    worst = 0.0
    for c in range(3):
        u = nodal_field(pat, mesh.coords[:, c])
        worst = max(worst, abs(float(u @ (S @ u)) - target) / target)
    return worst


def rigid_modes(mesh, pat):
    """The three translations and three infinitesimal rotations of the body (3 DOFs per node)."""
    xyz = mesh.coords
    modes = [nodal_field(pat, np.ones(mesh.nnodes), 3, d) for d in range(3)]
    for i, j in ((0, 1), (1, 2), (2, 0)):
        modes.append(nodal_field(pat, -xyz[:, j], 3, i) + nodal_field(pat, xyz[:, i], 3, j))
    return modes


def rigid_mode_defect(mesh, pat, vals):
    """max over modes and rows |(K u)_i| / (|K| |u|)_i."""
    S = csr(pat, vals)
    A = abs(S)
    worst = 0.0
    for u in rigid_modes(mesh, pat):
        worst = max(worst, float(np.max(np.abs(S @ u) / np.maximum(A @ np.abs(u), 1e-300))))
    return worst


def scaled_residual(pat, vals, b, x):
    """||D (b - A x)|| / ||D b|| with D = 1/sqrt(|diag A|): the relative residual of the scaled
    system D A D (D^-1 x) = D b, which the stopping test of a scaled solve bounds by its tolerance."""
    S = csr(pat, vals)
    d = np.abs(S.diagonal())
    D = np.where(d > 0, 1.0 / np.sqrt(np.where(d > 0, d, 1.0)), 1.0)
    r = b - S @ x
    return float(np.linalg.norm(D * r) / np.linalg.norm(D * b))
