"""ctypes binding of the CPU oracle (oracle/elmer_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py as the checker.  The product library never loads it.
All index arrays are 1-based int32, as in Elmer's Matrix_t.

Pinned to the reference's own regression targets (the heateq and linearsolvers NRM values
on their committed 2D mesh, tests/golden/) and to independent transcriptions of the
reference's loops; not pinned against a built ElmerSolver, which is Fortran and cannot be
built here.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libelmer_oracle.so")
_lib = None

CG, BICGSTAB, GCR, BICGSTABL = 1, 2, 3, 4
PREC_NONE, PREC_DIAGONAL, PREC_ILU0, PREC_ILUT = 0, 1, 2, 3

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class _Params(C.Structure):
    _fields_ = [("method", C.c_int), ("precond", C.c_int), ("max_iter", C.c_int),
                ("tol", C.c_double), ("scale_system", C.c_int), ("omp_threads", C.c_int),
                ("ilu_order", C.c_int), ("restart", C.c_int), ("ilut_tol", C.c_double), ("divtol", C.c_double),
                ("blas_threads", C.c_int), ("block_starts", C.c_void_p), ("nblocks", C.c_int)]


class _Result(C.Structure):
    _fields_ = [("info", C.c_int), ("iters", C.c_int), ("residual", C.c_double),
                ("seconds_solve", C.c_double), ("seconds_precond_setup", C.c_double)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def use_native() -> str:
    """Switch to the -march=native build of the same source (the timed CPU baseline), built for
    this host; call before the first oracle call.  Returns the library's path."""
    global _LIB_PATH
    if _lib is not None:
        raise RuntimeError("oracle already loaded")
    import hashlib

    try:  # one directory per host CPU (model and feature flags)
        info = [l for l in open("/proc/cpuinfo") if l.startswith(("model name", "flags"))][:2]
    except OSError:
        info = [os.uname().machine]
    tag = hashlib.sha1("".join(info).encode()).hexdigest()[:12]
    out = os.path.join(_HERE, "_build", "native_" + tag)
    subprocess.run(["make", "-s", "-C", _HERE, "native", "NATIVE_OUT=" + out], check=True)
    _LIB_PATH = os.path.join(out, "libelmer_oracle.so")
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_pattern_create.restype = C.c_void_p
        L.orc_pattern_create.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, C.c_int, C.c_int, C.c_int]
        L.orc_pattern_info.argtypes = [C.c_void_p] + [C.c_void_p] * 6
        L.orc_pattern_copy.argtypes = [C.c_void_p, _i32p, _i32p, _i32p, _i32p]
        L.orc_pattern_free.argtypes = [C.c_void_p]
        L.orc_assemble_poisson.argtypes = [C.c_int, _f64p, C.c_int, C.c_int, C.c_int, _i32p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, _i32p, C.c_int,
                                           _i32p, _i32p, _i32p, _f64p, _f64p]
        L.orc_assemble_elastic.argtypes = [C.c_int, _f64p, C.c_int, C.c_int, _i32p, C.c_double,
                                           C.c_double, _f64p, _i32p, C.c_int, _i32p, _i32p,
                                           _i32p, _f64p, _f64p]
        L.orc_dirichlet.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f64p, _f64p, C.c_int, _i32p,
                                    _f64p, C.c_int, C.c_int]
        L.orc_solve.restype = C.c_int
        L.orc_solve.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f64p, _f64p, _f64p,
                                C.POINTER(_Params), C.POINTER(_Result)]
        L.orc_spmv.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int]
        L.orc_ilu0.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f64p, _f64p]
        L.orc_lusolve.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f64p, _f64p]
        L.orc_ilu_pattern.restype = C.c_longlong
        L.orc_ilu_pattern.argtypes = [C.c_int, _i32p, _i32p, _i32p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
        L.orc_iluk.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _i32p, _f64p]
        L.orc_ilut.restype = C.c_longlong
        L.orc_ilut.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_double, C.c_longlong, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]
        L.orc_scale.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f64p, C.c_void_p, C.c_void_p,
                                _f64p, C.POINTER(C.c_double), C.c_int]
        L.orc_compute_norm.restype = C.c_double
        L.orc_compute_norm.argtypes = [C.c_int, _f64p]
        L.orc_lower_levels.restype = C.c_int
        L.orc_lower_levels.argtypes = [C.c_int, _i32p, _i32p, _i32p, _i32p]
        _lib = L
    return _lib


@dataclass
class Pattern:
    n: int
    nnz: int
    dofs: int
    perm: np.ndarray
    rows: np.ndarray
    cols: np.ndarray
    diag: np.ndarray
    hbw_before: int
    hbw_after: int
    start_node: int
    rejected: int


def _ptr(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data


def create_pattern(mesh, dofs: int = 1, optimize: bool = True, use_always: bool = False) -> Pattern:
    L = lib()
    el = np.ascontiguousarray(mesh.elements, dtype=np.int32)
    h = L.orc_pattern_create(mesh.nnodes, el.shape[0], el.shape[1], el, dofs, int(optimize), int(use_always))
    n, nnz = C.c_int(), C.c_longlong()
    hb, ha, st, rj = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    L.orc_pattern_info(h, C.byref(n), C.byref(nnz), C.byref(hb), C.byref(ha), C.byref(st), C.byref(rj))
    perm = np.zeros(mesh.nnodes, np.int32)
    rows = np.zeros(n.value + 1, np.int32)
    cols = np.zeros(nnz.value, np.int32)
    diag = np.zeros(n.value, np.int32)
    L.orc_pattern_copy(h, perm, rows, cols, diag)
    L.orc_pattern_free(h)
    return Pattern(n.value, nnz.value, dofs, perm, rows, cols, diag, hb.value, ha.value, st.value, rj.value)


def assemble_poisson(mesh, pat: Pattern, elem_k=None, nodal_k=None, load=None, cdim=None):
    L = lib()
    values = np.zeros(pat.nnz, np.float64)
    rhs = np.zeros(pat.n, np.float64)
    xyz = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    if cdim is None:
        cdim = 2 if mesh.elem_code // 100 <= 4 else 3
    keep = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None for a in (elem_k, nodal_k, load)]
    L.orc_assemble_poisson(mesh.nnodes, xyz, cdim, mesh.nelem, mesh.elem_code,
                           np.ascontiguousarray(mesh.elements, np.int32),
                           *[None if a is None else a.ctypes.data for a in keep],
                           pat.perm, pat.n, pat.rows, pat.cols, pat.diag, values, rhs)
    return values, rhs


def assemble_elastic(mesh, pat: Pattern, young: float, poisson: float, body_force):
    L = lib()
    values = np.zeros(pat.nnz, np.float64)
    rhs = np.zeros(pat.n, np.float64)
    L.orc_assemble_elastic(mesh.nnodes, np.ascontiguousarray(mesh.coords, np.float64), mesh.nelem,
                           mesh.elem_code, np.ascontiguousarray(mesh.elements, np.int32),
                           young, poisson, np.asarray(body_force, np.float64), pat.perm, pat.n,
                           pat.rows, pat.cols, pat.diag, values, rhs)
    return values, rhs


def dirichlet(pat: Pattern, values, rhs, con_rows, con_vals=None, symmetric=False, scale=True):
    con_rows = np.ascontiguousarray(con_rows, np.int32)
    if con_vals is None:
        con_vals = np.zeros(con_rows.size, np.float64)
    lib().orc_dirichlet(pat.n, pat.rows, pat.cols, pat.diag, values, rhs, con_rows.size, con_rows,
                        np.ascontiguousarray(con_vals, np.float64), int(symmetric), int(scale))


def solve(pat: Pattern, values, b, method=BICGSTAB, precond=PREC_ILU0, max_iter=1000, tol=1e-10,
          x0=None, scale=True, threads=0, ilu_order=0, restart=0, ilut_tol=0.0, divtol=0.0, blas_threads=0,
          block_starts=None):
    """orc_solve.  threads: SpMV threads (0: all); blas_threads: threads for the vector operations
    (0: serial as the reference's netlib BLAS, the checker's setting; > 0 for the timed baseline);
    block_starts (0-based row offsets of a partition, nblocks + 1 entries): block-Jacobi ILU0."""
    x = np.zeros(pat.n) if x0 is None else np.array(x0, dtype=np.float64)
    bst = None if block_starts is None else np.ascontiguousarray(block_starts, np.int32)
    p = _Params(method, precond, max_iter, tol, int(scale), threads, ilu_order, restart, ilut_tol, divtol,
                blas_threads, None if bst is None else bst.ctypes.data, 0 if bst is None else len(bst) - 1)
    r = _Result()
    lib().orc_solve(pat.n, pat.rows, pat.cols, pat.diag, np.ascontiguousarray(values, np.float64),
                    np.ascontiguousarray(b, np.float64), x, C.byref(p), C.byref(r))
    return x, {"info": r.info, "iters": r.iters, "residual": r.residual,
               "seconds": r.seconds_solve, "seconds_precond_setup": r.seconds_precond_setup}


def spmv(pat: Pattern, values, u, threads=0):
    v = np.zeros(pat.n)
    lib().orc_spmv(pat.n, pat.rows, pat.cols, np.ascontiguousarray(values, np.float64),
                   np.ascontiguousarray(u, np.float64), v, threads)
    return v


def ilu0(pat: Pattern, values):
    out = np.zeros(pat.nnz)
    lib().orc_ilu0(pat.n, pat.rows, pat.cols, pat.diag, np.ascontiguousarray(values, np.float64), out)
    return out


def ilu_pattern(pat: Pattern, order: int):
    """ILU(order) structure (1-based rows, cols, diag): InitializeILU1 applied order times."""
    nz = lib().orc_ilu_pattern(pat.n, pat.rows, pat.cols, pat.diag, order, 0, None, None, None)
    r, c, d = np.zeros(pat.n + 1, np.int32), np.zeros(nz, np.int32), np.zeros(pat.n, np.int32)
    lib().orc_ilu_pattern(pat.n, pat.rows, pat.cols, pat.diag, order, nz, r.ctypes.data, c.ctypes.data,
                          d.ctypes.data)
    return r, c, d


def iluk(pat: Pattern, values, order: int):
    """ILU(order) factors on its structure; returns (rows, cols, diag, values), 1-based."""
    r, c, d = ilu_pattern(pat, order)
    out = np.zeros(c.size)
    lib().orc_iluk(pat.n, pat.rows, pat.cols, np.ascontiguousarray(values, np.float64), r, c, d, out)
    return r, c, d, out


def ilut(pat: Pattern, values, tol: float):
    """CRS_ILUT factors (threshold ILU): (rows, cols, diag, values), 1-based, inverted U diagonal."""
    v = np.ascontiguousarray(values, np.float64)
    nz = lib().orc_ilut(pat.n, pat.rows, pat.cols, v, float(tol), 0, None, None, None, None)
    if nz < 0:
        raise ValueError("ILUT: a row's diagonal is missing")
    r, c, d, out = np.zeros(pat.n + 1, np.int32), np.zeros(nz, np.int32), np.zeros(pat.n, np.int32), np.zeros(nz)
    lib().orc_ilut(pat.n, pat.rows, pat.cols, v, float(tol), nz, r.ctypes.data, c.ctypes.data, d.ctypes.data,
                   out.ctypes.data)
    return r, c, d, out


def lusolve_on(rows, cols, diag, ilu, b):
    """CRS_LUPrecondition on a factor with its own structure (ILU(n), ILUT), 1-based arrays."""
    x = np.array(b, dtype=np.float64)
    lib().orc_lusolve(len(diag), np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32),
                      np.ascontiguousarray(diag, np.int32), np.ascontiguousarray(ilu, np.float64), x)
    return x


def lusolve(pat: Pattern, ilu, b):
    x = np.array(b, dtype=np.float64)
    lib().orc_lusolve(pat.n, pat.rows, pat.cols, pat.diag, np.ascontiguousarray(ilu, np.float64), x)
    return x


def scale(pat: Pattern, values, b=None, x=None, rhs_scale=True):
    """In-place ScaleLinearSystem; returns (DiagScaling, RhsScaling)."""
    D = np.zeros(pat.n)
    rs = C.c_double()
    lib().orc_scale(pat.n, pat.rows, pat.cols, pat.diag, values,
                    None if b is None else b.ctypes.data, None if x is None else x.ctypes.data,
                    D, C.byref(rs), int(rhs_scale))
    return D, rs.value


def compute_norm(x):
    x = np.ascontiguousarray(x, np.float64)
    return lib().orc_compute_norm(x.size, x)


def lower_levels(pat: Pattern):
    lv = np.zeros(pat.n, np.int32)
    nl = lib().orc_lower_levels(pat.n, pat.rows, pat.cols, pat.diag, lv)
    return nl, lv
