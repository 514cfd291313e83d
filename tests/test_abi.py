"""C-ABI surface: the library loads and exports every declared symbol; keyword parsing (CPU)."""
import ctypes as C
import os

import numpy as np
import pytest

import elmerfem_b200 as eg
from elmerfem_b200 import _lib


def test_library_loads_and_exports_declared_symbols():
    L = _lib.lib()
    declared = _lib.declared_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared) == set(_lib.PROTOTYPES), set(declared) ^ set(_lib.PROTOTYPES)


def test_params_default_matches_elmer_defaults():
    p = _lib.Params()
    _lib.lib().egpu_params_default(C.byref(p), eg.CG, eg.PREC_DIAGONAL)
    assert (p.method, p.precond, p.scale_system, p.refactorize, p.precond_recompute) == (1, 1, 1, 1, 1)


def test_create_on_missing_device_fails_cleanly():
    h = C.c_void_p()
    rc = _lib.lib().egpu_create(10_000, C.byref(h))
    assert rc == -2 and not h.value


def test_null_arguments_rejected():
    raw = C.CDLL(_lib.LIB_PATH)  # untyped view: pass NULLs straight through
    assert raw.egpu_iter_solve(None, None, None, None, None) == -1
    assert raw.egpu_iter_solve_dev(None, None, None, None, None) == -1
    assert raw.egpu_assembly_bind(None, 0, None, 3, 0, 808, None, None, 1) == -1
    assert raw.egpu_matrix_bind(None, 0, None, None, None, None, None) == -1
    assert raw.egpu_mv(None, None, None) == -1


SIF = """
Solver 1
  Equation = "Heat Equation"
  Linear System Solver = "Iterative"
  Linear System Iterative Method = "BiCGStab"
  Linear System Max Iterations = 350
  Linear System Convergence Tolerance = 1.0e-08
  Linear System Abort Not Converged = True
  Linear System Preconditioning = "ILU0"
  Linear System Residual Output = 1
End
"""


def test_sif_keywords():
    p = eg.SolverParams.from_sif(SIF)
    assert (p.method, p.precond, p.max_iter, p.tol) == (eg.BICGSTAB, eg.PREC_ILU0, 350, 1e-8)
    assert p.scale_system and p.abort_not_converged
    q = eg.SolverParams.from_sif({"Linear System Iterative Method": "CG", "Linear System Preconditioning": "Diagonal",
                                  "Linear System Max Iterations": 10, "Linear System Convergence Tolerance": 1e-6,
                                  "Linear System Symmetric": True, "Linear System Precision": "mixed"})
    assert (q.method, q.precond, q.symmetric, q.precision) == (eg.CG, eg.PREC_DIAGONAL, True, eg.MIXED)


def test_sif_gcr_bicgstabl():
    base = {"Linear System Max Iterations": 100, "Linear System Convergence Tolerance": 1e-8}
    p = eg.SolverParams.from_sif(dict(base, **{"Linear System Iterative Method": "GCR",
                                               "Linear System GCR Restart": 20}))
    assert (p.method, p.restart) == (eg.GCR, 20)
    q = eg.SolverParams.from_sif(dict(base, **{"Linear System Iterative Method": "BiCGStabl",
                                               "BiCGstabl polynomial degree": 4}))
    assert (q.method, q.restart) == (eg.BICGSTABL, 4)
    assert eg.SolverParams.from_sif(dict(base, **{"Linear System Iterative Method": "BiCGStabl"})).restart == 0
    # Linear System Divergence Tolerance (IterSolve.src:364-366): absent -> no bound (0 here, HUGE there)
    assert p.divtol == 0.0 and p.to_c().divtol == 0.0
    d = eg.SolverParams.from_sif(dict(base, **{"Linear System Iterative Method": "GCR",
                                               "Linear System Divergence Tolerance": 1e4}))
    assert d.divtol == 1e4 and d.to_c().divtol == 1e4
    with pytest.raises(ValueError):
        eg.SolverParams.from_sif(dict(base, **{"Linear System Iterative Method": "BiCGStabl",
                                               "BiCGstabl polynomial degree": 1}))


def test_sif_ilu_order():
    base = {"Linear System Max Iterations": 10, "Linear System Convergence Tolerance": 1e-6}
    assert eg.SolverParams.from_sif(dict(base, **{"Linear System Preconditioning": "ILU2"})).ilu_order == 2
    p = eg.SolverParams.from_sif(dict(base, **{"Linear System Preconditioning": "ILU",
                                               "Linear System ILU Order": 1}))
    assert (p.precond, p.ilu_order) == (eg.PREC_ILU0, 1)
    assert eg.SolverParams.from_sif(dict(base, **{"Linear System Preconditioning": "ILU0"})).ilu_order == 0


def test_sif_ilut():
    base = {"Linear System Max Iterations": 10, "Linear System Convergence Tolerance": 1e-6}
    p = eg.SolverParams.from_sif(dict(base, **{"Linear System Preconditioning": "ILUT",
                                               "Linear System ILUT Tolerance": 1e-3}))
    assert (p.precond, p.ilut_tol, p.ilu_order) == (eg.PREC_ILUT, 1e-3, 0)
    # absent tolerance: 0 (ListGetCReal's default), nothing dropped
    assert eg.SolverParams.from_sif(dict(base, **{"Linear System Preconditioning": "ILUT"})).ilut_tol == 0.0
    assert p.to_c().ilut_tol == 1e-3
    with pytest.raises(ValueError):
        eg.SolverParams.from_sif(dict(base, **{"Linear System Preconditioning": "ILUT",
                                               "Linear System ILUT Tolerance": -1}))


@pytest.mark.parametrize("bad", [{"Linear System Solver": "Direct"}, {"Linear System Iterative Method": "GMRES"},
                                 {"Linear System Preconditioning": "BILU1"}])
def test_sif_outside_the_path(bad):
    kw = {"Linear System Max Iterations": 10, "Linear System Convergence Tolerance": 1e-6}
    kw.update(bad)
    with pytest.raises(NotImplementedError):
        eg.SolverParams.from_sif(kw)


def test_sif_required_keywords():
    with pytest.raises(KeyError):
        eg.SolverParams.from_sif({"Linear System Convergence Tolerance": 1e-6})


def test_cache_queries_without_gpu():
    """The cache queries need no device while nothing is cached (no CUDA call is made)."""
    assert eg.cached_bytes() == 0 and eg.cached_bytes(0) == 0
    assert eg.release_cached_memory() == 0


def test_matvec_hook_without_a_device_returns_nan():
    """The Matrix Vector Proc hook has no status argument: when no device can take the product
    it fills v with NaN (the caller's Krylov method then cannot converge) and leaves the handle
    slot empty.
    Where a device exists the same call must give the product itself."""
    n = 3
    rows = np.array([1, 3, 6, 8], np.int32)
    cols = np.array([1, 2, 1, 2, 3, 2, 3], np.int32)
    vals = np.array([4.0, -1.0, -1.0, 4.0, -1.0, -1.0, 4.0])
    u = np.array([1.0, 2.0, 3.0])
    v = np.zeros(n)
    h = C.c_void_p()
    nn, zero = C.c_int(n), C.c_int(0)
    _lib.lib().egpu_matvec_subr(C.byref(h), C.byref(nn), rows, cols, vals, u, v, C.byref(zero))
    import torch

    if torch.cuda.is_available():
        assert np.allclose(v, [2.0, 4.0, 10.0])
    else:
        assert np.all(np.isnan(v)) and not h.value


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """No fallback: without the built library every entry point raises."""
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libelmergpu.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(eg.LibError, match="missing"):
        eg.Context(0)
    with pytest.raises(eg.LibError, match="missing"):
        eg.cached_bytes()


def test_plain_c_host_links_and_calls(tmp_path):
    """The ABI is plain C: a C99 program includes the header, links the library and calls it."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "host.c"
    src.write_text('#include "elmergpu.h"\n'
                   "int main(void) {\n"
                   "  egpu_params p;\n"
                   "  egpu_params_default(&p, EGPU_BICGSTAB, EGPU_PREC_ILU0);\n"
                   "  if (p.method != EGPU_BICGSTAB || p.precond != EGPU_PREC_ILU0) return 2;\n"
                   "  if (egpu_iter_solve(0, 0, 0, &p, 0) != EGPU_ERR_ARG) return 3;\n"
                   "  return egpu_cached_bytes(-1) == 0 ? 0 : 4;\n"
                   "}\n")
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "host"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(root, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lelmergpu", "-Wl,-rpath," + libdir], check=True, capture_output=True)
    assert subprocess.run([str(exe)]).returncode == 0
