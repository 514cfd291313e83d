"""B200-native ElmerSolver linear-system path: CRS assembly, SpMV, CG/BiCGStab, ILU0/Jacobi.

The compute lives in ``libelmergpu.so`` (CUDA, sm_100a) behind the C ABI declared in
``include/elmergpu.h``; this package is a thin host mirror of the reference's interface.
"""
from . import meshgen
from ._lib import BICGSTAB, BICGSTABL, CG, FP64, GCR, MIXED, PREC_DIAGONAL, PREC_ILU0, PREC_ILUT, PREC_NONE, LibError, build, lib
from .solver import (Batch, Context, CRSPattern, Matrix, NotConverged, SolverParams, cached_bytes, compute_norm,
                     create_matrix, iter_solver, parse_sif_section, release_cached_memory)

__all__ = ["meshgen", "BICGSTAB", "CG", "FP64", "MIXED", "PREC_DIAGONAL", "PREC_ILU0", "PREC_ILUT", "PREC_NONE", "LibError",
           "build", "lib", "Batch", "Context", "CRSPattern", "Matrix", "NotConverged", "SolverParams", "compute_norm",
           "create_matrix", "iter_solver", "parse_sif_section", "cached_bytes", "release_cached_memory"]
