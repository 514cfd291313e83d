"""Host-side mirror of ElmerSolver's linear-system interface over the C ABI.

Names follow the reference: ``create_matrix`` is CreateMatrix (ElementUtils.src:698),
``Matrix`` is a device-bound Matrix_t (Types.src:155-228), ``iter_solver`` is IterSolver
(IterSolve.src:144) with SolveLinearSystem's scaling around it (SolverUtils.src:7151), and
``SolverParams.from_sif`` reads the same keywords as IterSolver (IterSolve.src:221-420).
All compute runs in libelmergpu.so on the GPU; nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import re
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (BICGSTAB, BICGSTABL, CG, FP64, GCR, MIXED, PREC_DIAGONAL, PREC_ILU0, PREC_ILUT, PREC_NONE, LibError,
                   check, lib)


class NotConverged(RuntimeError):
    """Raised like Fatal('IterSolve', ...) when Linear System Abort Not Converged is True."""


class Context:
    """One GPU, one stream (egpu_create)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        check(lib().egpu_create(device, C.byref(self._h)), None, "egpu_create")
        self.device = device
        self._children = weakref.WeakSet()  # matrices bound to this context, freed before it

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        """cudaStream_t (as an integer) every call of this context runs on."""
        return int(lib().egpu_stream(self._h) or 0)

    @property
    def kernel_launches(self) -> int:
        return int(lib().egpu_kernel_launches(self._h))

    def set_wait_limit(self, seconds: float = 0.0):
        """Bound of every device-side wait of this context's kernels (0: the default 2 s)."""
        check(lib().egpu_set_wait_limit(self._h, float(seconds)), self._h, "egpu_set_wait_limit")

    def abort(self, raise_: bool = True):
        """Raise (or clear) the host-mapped abort word: the solve in flight and later ones
        return EGPU_ERR_ABORT until it is cleared.  Safe from any thread."""
        check(lib().egpu_abort(self._h, int(bool(raise_))), self._h, "egpu_abort")

    def wait_selftest(self, which: int) -> int:
        """Status recorded by a kernel whose bounded wait runs out by design (see the header)."""
        return int(lib().egpu_wait_selftest(self._h, int(which)))

    def close(self):
        if self._h:
            for child in list(self._children):
                child.free()
            lib().egpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class CRSPattern:
    """Rows/Cols/Diag (1-based, as Matrix_t) plus Perm (node -> row block)."""

    n: int
    nnz: int
    dofs: int
    perm: np.ndarray
    rows: np.ndarray
    cols: np.ndarray
    diag: np.ndarray


def create_matrix(mesh, dofs: int = 1, optimize_bandwidth: bool = True) -> CRSPattern:
    """CreateMatrix for a mesh whose nodes are all active (egpu_pattern_create)."""
    L = lib()
    el = np.ascontiguousarray(mesh.elements, dtype=np.int32)
    n, nnz = C.c_int(), C.c_longlong()
    check(L.egpu_pattern_create(mesh.nnodes, el.shape[0], el.shape[1], el, dofs, int(optimize_bandwidth),
                                C.byref(n), C.byref(nnz), None, None, None, None), None, "egpu_pattern_create")
    perm = np.zeros(mesh.nnodes, np.int32)
    rows = np.zeros(n.value + 1, np.int32)
    cols = np.zeros(nnz.value, np.int32)
    diag = np.zeros(n.value, np.int32)
    check(L.egpu_pattern_create(mesh.nnodes, el.shape[0], el.shape[1], el, dofs, int(optimize_bandwidth),
                                C.byref(n), C.byref(nnz), perm.ctypes.data, rows.ctypes.data,
                                cols.ctypes.data, diag.ctypes.data), None, "egpu_pattern_create")
    return CRSPattern(n.value, nnz.value, dofs, perm, rows, cols, diag)


@dataclass
class SolverParams:
    method: int = BICGSTAB
    precond: int = PREC_ILU0
    max_iter: int = 1000
    tol: float = 1e-10
    scale_system: bool = True
    precision: int = FP64
    refactorize: bool = True
    precond_recompute: int = 1
    inner_tol: float = 0.0        # 0: chosen by preconditioner (1e-2 Diagonal/none, 3e-2 ILU0)
    inner_max_iter: int = 2000
    max_refinements: int = 100
    abort_not_converged: bool = True
    symmetric: bool = False
    ilu_order: int = 0            # ILU(n) with precond PREC_ILU0 (Linear System ILU Order)
    restart: int = 0              # GCR restart (0: max_iter) / BiCGStab(l) degree (0: 2)
    ilut_tol: float = 0.0         # drop tolerance with precond PREC_ILUT (Linear System ILUT Tolerance)
    divtol: float = 0.0           # Linear System Divergence Tolerance (0: none); GCR and BiCGStab(l)
    ilu_sweeps: int = -1          # mixed BiCGStab + ILU0: Jacobi sweeps per triangle in the FP32 inner
                                  # solves (0: exact solves; < 0: measured against exact by the library)

    def to_c(self) -> _lib.Params:
        return _lib.Params(self.method, self.precond, self.max_iter, self.tol, int(self.scale_system),
                           self.precision, int(self.refactorize), self.precond_recompute, self.inner_tol,
                           self.inner_max_iter, self.max_refinements, self.ilu_order, self.restart,
                           float(self.ilut_tol), float(self.divtol), int(self.ilu_sweeps))

    @classmethod
    def from_sif(cls, keywords) -> "SolverParams":
        """Build from a Solver section (text or {keyword: value}); IterSolve.src:221-420."""
        kw = parse_sif_section(keywords) if isinstance(keywords, str) else {k.lower(): v for k, v in keywords.items()}
        solver = str(kw.get("linear system solver", "iterative")).lower()
        if solver != "iterative":
            raise NotImplementedError(f"Linear System Solver = {solver}: only 'iterative' is on this path")
        meth = str(kw.get("linear system iterative method", "bicgstab")).lower()
        methods = {"bicgstab": BICGSTAB, "cg": CG, "gcr": GCR, "bicgstabl": BICGSTABL}
        if meth not in methods:
            raise NotImplementedError(f"Linear System Iterative Method = {meth}")
        prec = str(kw.get("linear system preconditioning", "none")).lower()
        ilu_n = 0
        ilut_tol = 0.0
        if prec.startswith("none"):
            pc = PREC_NONE
        elif prec.startswith("diagonal"):
            pc = PREC_DIAGONAL
        elif prec.startswith("ilut"):
            # IterSolve.src:384-388: ListGetCReal returns 0 when the keyword is absent
            ilut_tol = float(kw.get("linear system ilut tolerance", 0.0))
            if not ilut_tol >= 0.0:
                raise ValueError(f"Linear System ILUT Tolerance {ilut_tol} < 0")
            pc = PREC_ILUT
        elif prec.startswith("ilu"):
            # IterSolve.src: "ILU<n>" or "ILU" with Linear System ILU Order
            order = kw.get("linear system ilu order")
            ilu_n = int(round(float(order))) if order is not None else (int(prec[3]) if len(prec) > 3 and prec[3].isdigit() else 0)
            if not 0 <= ilu_n <= 9:
                raise ValueError(f"ILU order {ilu_n} outside 0..9")
            pc = PREC_ILU0
        else:
            raise NotImplementedError(f"Linear System Preconditioning = {prec}")
        if "linear system max iterations" not in kw:
            raise KeyError("Linear System Max Iterations is required (ListGetInteger without default)")
        if "linear system convergence tolerance" not in kw:
            raise KeyError("Linear System Convergence Tolerance is required")
        restart = 0
        if meth == "gcr" and "linear system gcr restart" in kw:
            restart = int(kw["linear system gcr restart"])
        if meth == "bicgstabl" and "bicgstabl polynomial degree" in kw:
            restart = int(kw["bicgstabl polynomial degree"])
            if restart < 2:
                raise ValueError("BiCGstabl polynomial degree < 2")
        p = cls(method=methods[meth], precond=pc, restart=restart,
                ilu_order=ilu_n if pc == PREC_ILU0 else 0, ilut_tol=ilut_tol,
                divtol=float(kw.get("linear system divergence tolerance", 0.0)),
                max_iter=int(kw["linear system max iterations"]),
                tol=float(kw["linear system convergence tolerance"]),
                scale_system=_bool(kw.get("linear system scaling", True)),
                refactorize=_bool(kw.get("linear system refactorize", True)),
                precond_recompute=max(1, int(kw.get("linear system precondition recompute", 1))),
                abort_not_converged=_bool(kw.get("linear system abort not converged", True)),
                symmetric=_bool(kw.get("linear system symmetric", False)))
        prec_kw = str(kw.get("linear system precision", "double")).lower()
        if prec_kw in ("mixed", "single-double", "fp32/fp64"):
            p.precision = MIXED
        if "linear system inner tolerance" in kw:
            p.inner_tol = float(kw["linear system inner tolerance"])
        return p


def _bool(v) -> bool:
    if isinstance(v, str):
        return v.strip().lower() in ("true", "logical true", "1", "yes")
    return bool(v)


def parse_sif_section(text: str) -> dict:
    """Keyword = [type] value lines of one .sif section -> {lowercase keyword: value}."""
    out = {}
    for line in text.splitlines():
        line = line.split("!")[0].strip()
        if "=" not in line:
            continue
        key, val = (s.strip() for s in line.split("=", 1))
        key = re.sub(r"\(\d+\)$", "", key).strip().lower()
        val = re.sub(r"^(real|integer|logical|string)\s+", "", val, flags=re.I).strip().strip('"')
        out[key] = val
    return out


class Matrix:
    """A Matrix_t bound to the GPU (egpu_matrix_bind)."""

    def __init__(self, ctx: Context, pattern: CRSPattern, values=None):
        self.ctx = ctx
        self.pattern = pattern
        self.n = pattern.n
        self.nnz = pattern.nnz
        self._h = C.c_void_p()
        vals = None if values is None else np.ascontiguousarray(values, np.float64)
        check(lib().egpu_matrix_bind(ctx.handle, pattern.n, pattern.rows, pattern.cols, pattern.diag,
                                     None if vals is None else vals.ctypes.data, C.byref(self._h)),
              ctx.handle, "egpu_matrix_bind")
        ctx._children.add(self)

    @classmethod
    def clone(cls, proto: "Matrix") -> "Matrix":
        """A matrix sharing proto's pattern and bound mesh, with its own values (egpu_matrix_clone)."""
        obj = cls.__new__(cls)
        obj.ctx, obj.pattern, obj.n, obj.nnz = proto.ctx, proto.pattern, proto.n, proto.nnz
        obj._h = C.c_void_p()
        check(lib().egpu_matrix_clone(proto.handle, C.byref(obj._h)), proto.ctx.handle, "egpu_matrix_clone")
        proto.ctx._children.add(obj)
        return obj

    def footprint(self, precond: int) -> int:
        return int(lib().egpu_matrix_footprint(self._h, precond))

    @property
    def handle(self):
        return self._h

    def free(self):
        # a matrix must not outlive its context: Context.close() frees its matrices first
        if self._h and self.ctx._h:
            lib().egpu_matrix_free(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def update_values(self, values):
        check(lib().egpu_matrix_update_values(self._h, np.ascontiguousarray(values, np.float64)), self.ctx.handle,
              "egpu_matrix_update_values")

    def values(self) -> np.ndarray:
        v = np.zeros(self.nnz)
        check(lib().egpu_matrix_values_download(self._h, v), self.ctx.handle, "values")
        return v

    def rhs(self) -> np.ndarray:
        v = np.zeros(self.n)
        check(lib().egpu_matrix_rhs_download(self._h, v), self.ctx.handle, "rhs")
        return v

    def mv(self, u) -> np.ndarray:
        """Matrix Vector Proc: v = A u on the GPU."""
        v = np.zeros(self.n)
        check(lib().egpu_mv(self._h, np.ascontiguousarray(u, np.float64), v), self.ctx.handle, "egpu_mv")
        return v

    # ---- preconditioner state (A%ILUValues, A%DiagScaling)
    def prepare(self, params: "SolverParams | int"):
        """One-time preconditioner structures (ILU(n) fill and level schedules) before the first
        solve; params is a SolverParams or a preconditioner code (ILU order 0)."""
        if not isinstance(params, SolverParams):
            params = SolverParams(precond=int(params))
        prm = params.to_c()
        check(lib().egpu_matrix_prepare(self._h, C.byref(prm)), self.ctx.handle, "egpu_matrix_prepare")

    def ilu(self, order: int, scale_system: bool = True):
        """Factor ILU(order) on the device (egpu_ilu_build); returns ilu_factors()."""
        check(lib().egpu_ilu_build(self._h, int(scale_system), int(order)), self.ctx.handle, "egpu_ilu_build")
        return self.ilu_factors()

    def ilu_factors(self):
        """The current ILU factors on their structure: (rows, cols, diag 1-based, values)."""
        nz = check(lib().egpu_ilu_download(self._h, None, None, None, None), self.ctx.handle, "egpu_ilu_download")
        r, c, d, v = np.zeros(self.n + 1, np.int32), np.zeros(nz, np.int32), np.zeros(self.n, np.int32), np.zeros(nz)
        check(lib().egpu_ilu_download(self._h, r.ctypes.data, c.ctypes.data, d.ctypes.data, v.ctypes.data),
              self.ctx.handle, "egpu_ilu_download")
        return r, c, d, v

    def tri_info(self) -> dict:
        """The triangular-solve schedule of the matrix's ILU structure (after a factorisation)."""
        info = np.zeros(6, np.int32)
        check(lib().egpu_tri_info(self._h, info.ctypes.data), self.ctx.handle, "egpu_tri_info")
        return {"node_block": int(info[0]), "lower_levels": int(info[1]), "upper_levels": int(info[2]),
                "max_width": int(info[3]), "single_block_fp64": bool(info[4]), "single_block_fp32": bool(info[5])}

    def ilut(self, tol: float, scale_system: bool = True):
        """CRS_ILUT on the (scaled) matrix: (rows, cols, diag 1-based, values with inverted U diagonal)."""
        check(lib().egpu_ilut_build(self._h, int(scale_system), float(tol)), self.ctx.handle, "egpu_ilut_build")
        return self.ilu_factors()

    def ilu0(self, scale_system: bool = True):
        """Factor ILU0 on the device; returns (ILUValues with inverted U diagonal, DiagScaling)."""
        check(lib().egpu_ilu0_build(self._h, int(scale_system)), self.ctx.handle, "egpu_ilu0_build")
        ilu, d = np.zeros(self.nnz), np.zeros(self.n)
        check(lib().egpu_ilu0_download(self._h, ilu.ctypes.data, d.ctypes.data), self.ctx.handle, "egpu_ilu0_download")
        return ilu, d

    def lu_precondition(self, v) -> np.ndarray:
        """CRS_LUPrecondition with the device factors: u = (LU)^-1 v."""
        u = np.zeros(self.n)
        check(lib().egpu_lu_precondition(self._h, np.ascontiguousarray(v, np.float64), u), self.ctx.handle,
              "egpu_lu_precondition")
        return u

    # ---- assembly seam
    def bind_assembly(self, mesh, cdim: int | None = None):
        p = self.pattern
        if cdim is None:
            cdim = 2 if mesh.elem_code // 100 <= 4 else 3
        check(lib().egpu_assembly_bind(self._h, mesh.nnodes, np.ascontiguousarray(mesh.coords, np.float64), cdim,
                                       mesh.nelem, mesh.elem_code, np.ascontiguousarray(mesh.elements, np.int32),
                                       p.perm, p.dofs), self.ctx.handle, "egpu_assembly_bind")

    def assemble_poisson(self, elem_k=None, nodal_k=None, load=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (elem_k, nodal_k, load)]
        check(lib().egpu_assemble_poisson(self._h, *[None if a is None else a.ctypes.data for a in arrs]),
              self.ctx.handle, "egpu_assemble_poisson")

    def assemble_elastic(self, young: float, poisson: float, body_force):
        check(lib().egpu_assemble_elastic(self._h, young, poisson, np.asarray(body_force, np.float64)),
              self.ctx.handle, "egpu_assemble_elastic")

    def dirichlet(self, con_rows, con_vals=None, symmetric: bool = False):
        r = np.ascontiguousarray(con_rows, np.int32)
        v = None if con_vals is None else np.ascontiguousarray(con_vals, np.float64)
        check(lib().egpu_dirichlet(self._h, r.size, r.ctypes.data, None if v is None else v.ctypes.data,
                                   int(symmetric)), self.ctx.handle, "egpu_dirichlet")

    # ---- solve
    def solve(self, b=None, x0=None, params: SolverParams | None = None):
        """IterSolver on host vectors (b None: the assembled RHS).  Returns (x, result dict)."""
        params = params or SolverParams()
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        res = _lib.Result()
        prm = params.to_c()
        if b is None:
            b = self.rhs()
        rc = check(lib().egpu_iter_solve(self._h, np.ascontiguousarray(b, np.float64), x, C.byref(prm), C.byref(res)),
                   self.ctx.handle, "egpu_iter_solve")
        out = res.as_dict()
        out["status"] = _lib.HUTI.get(rc, str(rc))
        if params.abort_not_converged and rc != 1:
            raise NotConverged(f"IterSolve: failed convergence tolerances ({out['status']}, iters {out['iters']})")
        return x, out

    def solve_dev(self, b_ptr: int | None, x_ptr: int, params: SolverParams | None = None) -> dict:
        """IterSolver on device buffers (raw CUDA pointers; b_ptr None: the assembled RHS)."""
        params = params or SolverParams()
        res = _lib.Result()
        prm = params.to_c()
        rc = check(lib().egpu_iter_solve_dev(self._h, b_ptr, x_ptr, C.byref(prm), C.byref(res)), self.ctx.handle,
                   "egpu_iter_solve_dev")
        out = res.as_dict()
        out["status"] = _lib.HUTI.get(rc, str(rc))
        if params.abort_not_converged and rc != 1:
            raise NotConverged(f"IterSolve: failed convergence tolerances ({out['status']}, iters {out['iters']})")
        return out


def iter_solver(A: Matrix, b, x, params: SolverParams):
    """IterSolver(A, x, b, Solver): solves in place into x (numpy), returns the result dict."""
    sol, res = A.solve(b, x, params)
    x[...] = sol
    return res


def cached_bytes(device: int = -1) -> int:
    """Bytes of freed device blocks the library keeps for reuse (egpu_cached_bytes); all devices if device < 0."""
    return int(lib().egpu_cached_bytes(device))


def release_cached_memory(device: int = -1) -> int:
    """Frees the library's cached device blocks (egpu_release_cached_memory); returns the bytes released."""
    return int(lib().egpu_release_cached_memory(device))


def compute_norm(x) -> float:
    """ComputeNorm default (SolverUtils.src:4983-4988): sqrt(sum(x^2)/n)."""
    x = np.asarray(x, np.float64)
    return float(np.sqrt(np.sum(x * x) / x.size))


class Batch:
    """Many independent systems solved together in mixed precision (egpu_batch_*).

    Parameters are fixed per batch; systems are added as host Matrix_t arrays (the batch
    owns the device copy) or as device-resident Matrix objects (borrowed).  step() runs one
    refinement check plus one chunk of inner iterations and returns the slots that finished:
    the building block of the continuous-batching server.
    """

    def __init__(self, ctx: Context, params: SolverParams, chunk: int = 64):
        self.ctx = ctx
        self._h = C.c_void_p()
        prm = params.to_c()
        check(lib().egpu_batch_create(ctx.handle, C.byref(prm), C.byref(self._h)), ctx.handle, "egpu_batch_create")
        lib().egpu_batch_set_chunk(self._h, chunk)
        self.n = {}
        self._borrowed = {}
        ctx._children.add(self)

    def add(self, pattern: CRSPattern, values, rhs) -> int:
        sid = check(lib().egpu_batch_add(self._h, pattern.n, pattern.rows, pattern.cols, pattern.diag,
                                         np.ascontiguousarray(values, np.float64),
                                         np.ascontiguousarray(rhs, np.float64)), self.ctx.handle, "egpu_batch_add")
        self.n[sid] = pattern.n
        return sid

    def add_matrix(self, A: "Matrix", b_ptr: int | None = None) -> int:
        sid = check(lib().egpu_batch_add_matrix(self._h, A.handle, b_ptr), self.ctx.handle, "egpu_batch_add_matrix")
        self.n[sid] = A.n
        self._borrowed[sid] = A
        return sid

    def step(self) -> list:
        fin = (C.c_int * 512)()
        nf = C.c_int()
        check(lib().egpu_batch_step(self._h, C.cast(fin, C.c_void_p), C.byref(nf)), self.ctx.handle, "egpu_batch_step")
        return [fin[i] for i in range(nf.value)]

    def pending(self) -> int:
        return check(lib().egpu_batch_pending(self._h), self.ctx.handle, "egpu_batch_pending")

    def tune(self) -> dict:
        """egpu_batch_tune: picks chunk length, blocks per SM, rows per warp in the SpMV phases
        and triangular-solve participants by timing real steps of the resident systems;
        returns the kept configuration."""
        cfg = _lib.BatchConfig()
        check(lib().egpu_batch_tune(self._h, C.byref(cfg)), self.ctx.handle, "egpu_batch_tune")
        return cfg.as_dict()

    def set_config(self, cfg: dict):
        c = _lib.BatchConfig(**{k: cfg[k] for k, _ in _lib.BatchConfig._fields_})
        check(lib().egpu_batch_set_config(self._h, C.byref(c)), self.ctx.handle, "egpu_batch_set_config")

    def solve(self):
        check(lib().egpu_batch_solve(self._h, None), self.ctx.handle, "egpu_batch_solve")

    def last_launch_ms(self) -> float:
        """Device milliseconds of the latest batched launch (the team solver's, or the last chunk's)."""
        ms = C.c_double(0.0)
        check(lib().egpu_batch_last_launch(self._h, C.byref(ms)), self.ctx.handle, "egpu_batch_last_launch")
        return ms.value

    def result(self, sid: int) -> dict:
        r = _lib.Result()
        check(lib().egpu_batch_result(self._h, sid, C.byref(r)), self.ctx.handle, "egpu_batch_result")
        out = r.as_dict()
        out["status"] = _lib.HUTI.get(r.info, str(r.info))
        return out

    def solution(self, sid: int) -> np.ndarray:
        x = np.zeros(self.n[sid])
        check(lib().egpu_batch_solution(self._h, sid, x), self.ctx.handle, "egpu_batch_solution")
        return x

    def remove(self, sid: int):
        check(lib().egpu_batch_remove(self._h, sid), self.ctx.handle, "egpu_batch_remove")
        self.n.pop(sid, None)
        self._borrowed.pop(sid, None)

    def free(self):
        if self._h and self.ctx._h:
            lib().egpu_batch_free(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
