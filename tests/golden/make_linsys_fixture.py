"""Writes tests/golden/linsys_hex4_*.dat: a Linear System Save file set laid out as
ElmerSolver writes it (SaveLinearSystem, SolverUtils.src:8588-8662), for the loader tests.

The system is the oracle's 4^3 hex Poisson (log-normal element conductivity, seed 11, unit
source, zero Dirichlet on the x = 0 face, non-symmetric elimination).  The statements reproduced:

    _a.dat      WRITE(1,'(I0,A,I0,A)',ADVANCE='NO') i,' ',Cols(j),' ' ; WRITE(1,*) Values(j)
                (CRS_PrintMatrix, CRSMatrix.src:924-936)
    _b.dat      WRITE(1,'(I0,A)',ADVANCE='NO') i,' ' ; '0.0' when |b_i| <= TINY, else WRITE(1,*) b_i
                (CRS_PrintRHS, CRSMatrix.src:953-962)
    _perm.dat   WRITE(1,'(I0,A,I0)') i,' ',Perm(i)
    _sizes.dat  WRITE(1,*) NumberOfRows ; WRITE(1,*) SIZE(Values) ; WRITE(1,*) SIZE(Perm)

List-directed output of a REAL(dp) is written in the layout gfortran gives it: 17 significant
digits, fixed notation for 0.1 <= |x| < 1e16 and otherwise an exponent of three digits with its
sign (1.0000000000000000E-002); list-directed integers are right-aligned in 12 columns.  Both
round-trip every double, so the loaded system is the oracle's to the bit.

    python tests/golden/make_linsys_fixture.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def list_directed_real(x: float) -> str:
    x = float(x)
    if x == 0.0:
        return "   0.0000000000000000     "
    ax = abs(x)
    sign = "-" if x < 0 else " "
    if 0.1 <= ax < 1e16:
        before = max(0, math.floor(math.log10(ax)) + 1)
        s = f"{ax:.{17 - before}f}"
        if len(s.split(".")[0].lstrip("0")) > before and before > 0:  # rounding carried into a new digit
            s = f"{ax:.{16 - before}f}"
        return " " + sign + s + "     "
    mant, exp = f"{ax:.16E}".split("E")
    e = int(exp)
    return " " + sign + f"{mant}E{'-' if e < 0 else '+'}{abs(e):03d}"


def list_directed_int(i: int) -> str:
    return f"{int(i):12d}"


def system():
    import oracle
    from elmerfem_b200 import meshgen
    from helpers import poisson_problem

    m = meshgen.hex_cube(4)
    k = meshgen.lognormal_conductivity(m.nelem, 1.0, 11)
    p, _, _, v, b, _ = poisson_problem(m, elem_k=k, load=np.ones(m.nnodes), sym=False, bc_ids=[1])
    return p, v, b, oracle


def write(prefix, p, v, b):
    n = p.n
    with open(prefix + "_a.dat", "w") as f:
        for i in range(n):
            for j in range(p.rows[i] - 1, p.rows[i + 1] - 1):
                f.write(f"{i + 1} {p.cols[j]} " + list_directed_real(v[j]) + "\n")
    tiny = np.finfo(np.float64).tiny
    with open(prefix + "_b.dat", "w") as f:
        for i in range(n):
            f.write(f"{i + 1} " + ("0.0" if abs(b[i]) <= tiny else list_directed_real(b[i])) + "\n")
    with open(prefix + "_perm.dat", "w") as f:
        for i, q in enumerate(p.perm, start=1):
            f.write(f"{i} {int(q)}\n")
    with open(prefix + "_sizes.dat", "w") as f:
        f.write(list_directed_int(n) + "\n" + list_directed_int(p.nnz) + "\n" + list_directed_int(len(p.perm)) + "\n")


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(os.path.dirname(HERE)))
    p, v, b, _ = system()
    write(os.path.join(HERE, "linsys_hex4"), p, v, b)
    print("wrote", os.path.join(HERE, "linsys_hex4_*.dat"))
