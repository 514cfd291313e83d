"""Elmer's Linear System Save files (SaveLinearSystem, SolverUtils.src:8588-8662).

    <prefix>_a.dat      "i j a_ij" per stored entry, rows in order (CRS_PrintMatrix, CRSMatrix.src:877-943)
    <prefix>_b.dat      "i b_i" per row, "0.0" when |b_i| <= TINY (CRS_PrintRHS, CRSMatrix.src:945-960)
    <prefix>_sizes.dat  NumberOfRows, SIZE(Values)[, SIZE(Perm)] one per line
    <prefix>_perm.dat   "i Perm(i)" (only with Linear System Save Perm)

Indices are 1-based.  Reading rebuilds Matrix_t Rows/Cols/Diag from the entry order, so a
system saved by ElmerSolver can be bound with Matrix / egpu_matrix_bind unchanged.
"""
from __future__ import annotations

import os

import numpy as np

from .solver import CRSPattern

_TINY = np.finfo(np.float64).tiny


def save_linear_system(prefix: str, pattern: CRSPattern, values, rhs, perm=None) -> None:
    rows, cols = pattern.rows, pattern.cols
    n = pattern.n
    row_of = np.repeat(np.arange(1, n + 1), np.diff(rows))
    with open(prefix + "_a.dat", "w") as f:
        for i, j, v in zip(row_of, cols, np.asarray(values, np.float64)):
            f.write(f"{i} {j} {float(v)!r}\n")
    with open(prefix + "_b.dat", "w") as f:
        for i, v in enumerate(np.asarray(rhs, np.float64), start=1):
            f.write(f"{i} 0.0\n" if abs(v) <= _TINY else f"{i} {float(v)!r}\n")
    with open(prefix + "_sizes.dat", "w") as f:
        f.write(f"{n}\n{len(values)}\n")
        if perm is not None:
            f.write(f"{len(perm)}\n")
    if perm is not None:
        with open(prefix + "_perm.dat", "w") as f:
            for i, p in enumerate(perm, start=1):
                f.write(f"{i} {int(p)}\n")


def load_linear_system(prefix: str):
    """Returns (CRSPattern, values, rhs); the pattern's perm is the saved Perm or identity."""
    sizes = [int(float(t)) for t in open(prefix + "_sizes.dat").read().split()]
    n, nnz = sizes[0], sizes[1]
    a = np.loadtxt(prefix + "_a.dat", ndmin=2)
    if a.shape[0] != nnz:
        raise ValueError(f"{prefix}_a.dat has {a.shape[0]} entries, sizes file says {nnz}")
    ri = a[:, 0].astype(np.int64)
    if np.any(np.diff(ri) < 0):
        raise ValueError("entries are not in row order")
    cols = a[:, 1].astype(np.int32)
    values = a[:, 2].astype(np.float64)
    counts = np.bincount(ri, minlength=n + 1)[1:]
    rows = np.concatenate([[1], 1 + np.cumsum(counts)]).astype(np.int32)
    diag = np.zeros(n, np.int32)
    for i in range(n):
        seg = np.nonzero(cols[rows[i] - 1:rows[i + 1] - 1] == i + 1)[0]
        if seg.size:
            diag[i] = rows[i] + seg[0]
    b = np.loadtxt(prefix + "_b.dat", ndmin=2)
    rhs = np.zeros(n)
    rhs[b[:, 0].astype(np.int64) - 1] = b[:, 1]
    perm = np.arange(1, n + 1, dtype=np.int32)
    if os.path.exists(prefix + "_perm.dat") and len(sizes) > 2:
        pm = np.loadtxt(prefix + "_perm.dat", ndmin=2).astype(np.int32)
        perm = np.zeros(sizes[2], np.int32)
        perm[pm[:, 0] - 1] = pm[:, 1]
    return CRSPattern(n, nnz, 1, perm, rows, cols, diag), values, rhs
