"""CPU checks of the level-synchronous single-block ILU0 solve's schedule.

tests/cpu_model/cta_model.cpp replays the kernel's staging windows and ring-buffer index
arithmetic on the product's own plan (elmerfem_b200/csrc/egpu_tri_plan.h), with every
shared-memory cell tagged by its writer, and the result must equal a sequential
CRS_LUSolve (fem/src/CRSMatrix.src:3346-3363) bit for bit in both precisions.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle
from elmerfem_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "elmerfem_b200", "csrc")
SMEM_MAX = 200 * 1024   # the product's budget (egpu_tri_cta.cu)


@pytest.fixture(scope="module")
def model(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("cta_model") / "cta_model.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-shared", "-fPIC", "-I", CSRC, "-o", so,
                    os.path.join(HERE, "cpu_model", "cta_model.cpp")], check=True)
    lib = C.CDLL(so)
    P = np.ctypeslib.ndpointer
    lib.cta_model_check.argtypes = [C.c_int, P(np.int32), P(np.int32), P(np.int32), P(np.float64), P(np.float64),
                                    P(np.float64), P(np.float64), C.c_longlong, C.c_int, P(np.int32)]
    lib.cta_model_check.restype = C.c_int
    return lib


def _factors(p, seed):
    """0-based CRS with well-conditioned random factor values (unit-ish diagonal inverse)."""
    rows, cols, diag = p.rows - 1, p.cols - 1, p.diag - 1
    rng = np.random.Generator(np.random.PCG64(seed))
    vals = rng.uniform(-0.1, 0.1, size=p.nnz)
    vals[diag] = rng.uniform(0.5, 1.5, size=p.n)
    b = rng.uniform(-1, 1, size=p.n)
    return rows.astype(np.int32), cols.astype(np.int32), diag.astype(np.int32), vals, b


MESHES = {
    "hex10": lambda: oracle.create_pattern(meshgen.hex_cube(10)),
    "hex32": lambda: oracle.create_pattern(meshgen.hex_cube(32)),
    "tet12": lambda: oracle.create_pattern(meshgen.tet_cube(12)),
    "elastic8": lambda: oracle.create_pattern(meshgen.hex_cube(8), dofs=3),
    "hex6_unoptimized": lambda: oracle.create_pattern(meshgen.hex_cube(6), optimize=False),
}


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("v", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("budget", [SMEM_MAX, 24 * 1024], ids=["full", "small"])
def test_block_solve_model(model, name, v, budget):
    p = MESHES[name]()
    rows, cols, diag, vals, b = _factors(p, 7)
    zm, zr = np.zeros(p.n), np.zeros(p.n)
    info = np.zeros(16, np.int32)
    rc = model.cta_model_check(p.n, rows, cols, diag, vals, b, zm, zr, budget, v, info)
    assert rc == 0, (rc, info[:9])
    assert info[0] == 1                        # representable
    if budget == SMEM_MAX and name != "hex32":
        assert info[1] == 1                    # fits the product's budget
    if info[1]:
        assert 1 <= info[3] <= 8 and info[6] <= budget
        assert np.array_equal(zm, zr)          # bit for bit
        assert np.all(np.isfinite(zm))
