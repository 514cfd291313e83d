"""Loader and ctypes prototypes for libelmergpu.so (the C ABI in include/elmergpu.h).

The library is built in-tree (elmerfem_b200/csrc/Makefile).  There is no fallback: if the
shared object is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libelmergpu.so")
CSRC = os.path.join(HERE, "csrc")
HEADER = os.path.join(os.path.dirname(HERE), "include", "elmergpu.h")

EGPU_OK = 0
ERRORS = {-1: "EGPU_ERR_ARG", -2: "EGPU_ERR_CUDA", -3: "EGPU_ERR_ALLOC", -4: "EGPU_ERR_TIMEOUT",
          -5: "EGPU_ERR_STATE", -6: "EGPU_ERR_BUDGET", -7: "EGPU_ERR_ABORT"}
HUTI = {1: "HUTI_CONVERGENCE", 2: "HUTI_MAXITER", 3: "HUTI_DIVERGENCE", 20: "HUTI_CG_RHO", 35: "HUTI_BICGSTAB_RHO",
        36: "HUTI_BICGSTAB_SNORM", 37: "HUTI_BICGSTAB_OMEGA"}

CG, BICGSTAB, GCR, BICGSTABL = 1, 2, 3, 4
PREC_NONE, PREC_DIAGONAL, PREC_ILU0, PREC_ILUT = 0, 1, 2, 3
FP64, MIXED = 0, 1

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p


class Params(C.Structure):
    _fields_ = [("method", C.c_int), ("precond", C.c_int), ("max_iter", C.c_int), ("tol", C.c_double),
                ("scale_system", C.c_int), ("precision", C.c_int), ("refactorize", C.c_int),
                ("precond_recompute", C.c_int), ("inner_tol", C.c_double), ("inner_max_iter", C.c_int),
                ("max_refinements", C.c_int), ("ilu_order", C.c_int), ("restart", C.c_int),
                ("ilut_tol", C.c_double), ("divtol", C.c_double), ("ilu_sweeps", C.c_int)]


class Result(C.Structure):
    _fields_ = [("info", C.c_int), ("iters", C.c_int), ("refinements", C.c_int), ("residual", C.c_double),
                ("seconds", C.c_double), ("seconds_setup", C.c_double), ("seconds_krylov", C.c_double),
                ("krylov_launches", C.c_int), ("precision_used", C.c_int), ("ilu_sweeps_used", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchConfig(C.Structure):
    _fields_ = [("chunk_iters", C.c_int), ("blocks_per_sm", C.c_int), ("tri_mult", C.c_int),
                ("candidates", C.c_int), ("rate", C.c_double), ("slices_per_warp", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("queued", C.c_longlong), ("resident", C.c_longlong), ("done", C.c_longlong),
                ("steps", C.c_longlong), ("used_bytes", C.c_double), ("seconds_prepare", C.c_double),
                ("seconds_step", C.c_double), ("seconds_retire", C.c_double), ("kernel_launches", C.c_longlong),
                ("bytes_h2d", C.c_double), ("bytes_d2h", C.c_double), ("requeues", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LibError(RuntimeError):
    """A negative status from the library; .code holds it (EGPU_ERR_*)."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


_lib = None

# name -> (restype, argtypes)
PROTOTYPES = {
    "egpu_params_default": (None, [C.POINTER(Params), C.c_int, C.c_int]),
    "egpu_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "egpu_destroy": (None, [_vp]),
    "egpu_last_error": (C.c_char_p, [_vp]),
    "egpu_kernel_launches": (C.c_longlong, [_vp]),
    "egpu_stream": (C.c_void_p, [_vp]),
    "egpu_set_wait_limit": (C.c_int, [_vp, C.c_double]),
    "egpu_abort": (C.c_int, [_vp, C.c_int]),
    "egpu_wait_selftest": (C.c_int, [_vp, C.c_int]),
    "egpu_cached_bytes": (C.c_longlong, [C.c_int]),
    "egpu_release_cached_memory": (C.c_longlong, [C.c_int]),
    "egpu_pattern_create": (C.c_int, [C.c_int, C.c_int, C.c_int, _i32p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_longlong), _vp, _vp, _vp, _vp]),
    "egpu_matrix_bind": (C.c_int, [_vp, C.c_int, _i32p, _i32p, _i32p, _vp, C.POINTER(_vp)]),
    "egpu_matrix_update_values": (C.c_int, [_vp, _f64p]),
    "egpu_matrix_values_download": (C.c_int, [_vp, _f64p]),
    "egpu_matrix_rhs_download": (C.c_int, [_vp, _f64p]),
    "egpu_matrix_free": (None, [_vp]),
    "egpu_matrix_clone": (C.c_int, [_vp, C.POINTER(_vp)]),
    "egpu_matrix_footprint": (C.c_longlong, [_vp, C.c_int]),
    "egpu_matrix_prepare": (C.c_int, [_vp, C.POINTER(Params)]),
    "egpu_ilu_pattern": (C.c_longlong, [C.c_int, _i32p, _i32p, _i32p, C.c_int, C.c_longlong, _vp, _vp, _vp]),
    "egpu_ilu_download": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "egpu_tri_info": (C.c_int, [_vp, _vp]),
    "egpu_ilut_build": (C.c_int, [_vp, C.c_int, C.c_double]),
    "egpu_iter_solve": (C.c_int, [_vp, _f64p, _f64p, C.POINTER(Params), C.POINTER(Result)]),
    "egpu_iter_solve_dev": (C.c_int, [_vp, _vp, _vp, C.POINTER(Params), C.POINTER(Result)]),
    "egpu_mv": (C.c_int, [_vp, _f64p, _f64p]),
    "egpu_mv_dev": (C.c_int, [_vp, _vp, _vp]),
    "egpu_matvec_subr": (None, [C.POINTER(_vp), C.POINTER(C.c_int), _i32p, _i32p, _f64p, _f64p, _f64p,
                                C.POINTER(C.c_int)]),
    "egpu_assembly_bind": (C.c_int, [_vp, C.c_int, _f64p, C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int]),
    "egpu_assemble_poisson": (C.c_int, [_vp, _vp, _vp, _vp]),
    "egpu_assemble_elastic": (C.c_int, [_vp, C.c_double, C.c_double, _f64p]),
    "egpu_dirichlet": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int]),
    "egpu_ilu0_build": (C.c_int, [_vp, C.c_int]),
    "egpu_ilu_build": (C.c_int, [_vp, C.c_int, C.c_int]),
    "egpu_ilu0_download": (C.c_int, [_vp, _vp, _vp]),
    "egpu_lu_precondition": (C.c_int, [_vp, _f64p, _f64p]),
    "egpu_lu_precondition_dev": (C.c_int, [_vp, _vp, _vp]),
    "egpu_cg_noalloc": (C.c_int, [C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(Params),
                                  C.POINTER(Result)]),
    "egpu_batch_create": (C.c_int, [_vp, C.POINTER(Params), C.POINTER(_vp)]),
    "egpu_batch_add": (C.c_int, [_vp, C.c_int, _i32p, _i32p, _i32p, _f64p, _f64p]),
    "egpu_batch_add_matrix": (C.c_int, [_vp, _vp, _vp]),
    "egpu_batch_set_chunk": (C.c_int, [_vp, C.c_int]),
    "egpu_batch_set_latency_mode": (C.c_int, [_vp, C.c_int]),
    "egpu_batch_step": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
    "egpu_batch_pending": (C.c_int, [_vp]),
    "egpu_batch_solve": (C.c_int, [_vp, _vp]),
    "egpu_batch_last_launch": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "egpu_batch_result": (C.c_int, [_vp, C.c_int, C.POINTER(Result)]),
    "egpu_batch_solution": (C.c_int, [_vp, C.c_int, _f64p]),
    "egpu_batch_remove": (C.c_int, [_vp, C.c_int]),
    "egpu_batch_tune": (C.c_int, [_vp, C.POINTER(BatchConfig)]),
    "egpu_batch_set_config": (C.c_int, [_vp, C.POINTER(BatchConfig)]),
    "egpu_batch_free": (None, [_vp]),
    "egpu_server_create": (C.c_int, [C.c_int, C.POINTER(Params), C.c_double, C.c_int, C.c_int, C.POINTER(_vp)]),
    "egpu_server_pattern": (C.c_int, [_vp, C.c_int, _i32p, _i32p, _i32p, C.POINTER(C.c_int)]),
    "egpu_server_pattern_mesh": (C.c_int, [_vp, C.c_int, C.c_int, _f64p, C.c_int, C.c_int, C.c_int, _i32p, _i32p,
                                           C.c_int]),
    "egpu_server_submit": (C.c_int, [_vp, C.c_int, _f64p, _f64p, C.POINTER(C.c_longlong)]),
    "egpu_server_submit_poisson": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_int, _vp, C.c_int,
                                             C.POINTER(C.c_longlong)]),
    "egpu_server_poll": (C.c_int, [_vp, C.c_longlong, _vp, C.POINTER(Result)]),
    "egpu_server_wait": (C.c_int, [_vp, C.c_longlong, C.c_double, _vp, C.POINTER(Result)]),
    "egpu_server_info": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "egpu_server_free": (None, [_vp]),
}


def build(force: bool = False) -> str:
    """Compile the CUDA library in-tree (nvcc, sm_100a)."""
    args = ["make", "-s", "-C", CSRC, "-j4"]
    if force:
        subprocess.run(["make", "-s", "-C", CSRC, "clean"], check=True)
    subprocess.run(args, check=True)
    return LIB_PATH


def declared_symbols() -> list[str]:
    """Every function name declared in include/elmergpu.h."""
    import re

    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(egpu_[a-z0-9_]+)\s*\(", text)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LibError(f"{LIB_PATH} is missing: build it with elmerfem_b200._lib.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, ctx=None, what: str = "") -> int:
    if rc < 0:
        msg = ERRORS.get(rc, str(rc))
        if ctx is not None:
            detail = lib().egpu_last_error(ctx)
            if detail:
                msg += ": " + detail.decode(errors="replace")
        raise LibError(f"{what}: {msg}", rc)
    return rc
