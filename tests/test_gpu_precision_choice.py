"""A mixed-precision CG / BiCGStab request runs the faster of the two paths measured on the
matrix itself: the first two mixed requests run mixed, the next run the FP64 drop-in until two
FP64 solves have run (the caller's own included), and from then on the drop-in is taken when
its latest time is below 0.85 of the latest mixed one.  Each path's first solve (one-time
set-up) is not compared.  The measurements outlive value updates.  Every solution meets 1e-8
against the oracle; EGPU_MIXED_AUTO=0 keeps the mixed path."""
import pytest

import elmerfem_b200 as eg
import oracle
from elmerfem_b200 import meshgen
from helpers import elastic_problem, rel

pytestmark = pytest.mark.gpu


def _params(precision, method=eg.BICGSTAB):
    return eg.SolverParams(method=method, precond=eg.PREC_ILU0, tol=1e-8, max_iter=5000, precision=precision)


class Model:
    """the library's bookkeeping, restated: counts and latest warm times per path"""

    def __init__(self):
        self.n = {eg.FP64: 0, eg.MIXED: 0}
        self.t = {eg.FP64: 0.0, eg.MIXED: 0.0}

    def expect(self):
        if self.n[eg.MIXED] < 2:
            return eg.MIXED
        if self.n[eg.FP64] < 2:
            return eg.FP64
        return eg.FP64 if self.t[eg.FP64] < 0.85 * self.t[eg.MIXED] else eg.MIXED

    def record(self, path, r):
        assert r["info"] == 1
        if self.n[path] > 0:
            self.t[path] = r["seconds"]
        self.n[path] += 1


def test_mixed_request_takes_the_measured_faster_path(ctx, monkeypatch):
    p, _, _, v, b, _ = elastic_problem(meshgen.hex_cube(8))
    x_orc, r_orc = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, tol=1e-8, max_iter=5000)
    A = eg.Matrix(ctx, eg.CRSPattern(p.n, p.nnz, 3, p.perm, p.rows, p.cols, p.diag), v)
    try:
        mod = Model()
        seen = []
        for _ in range(7):
            want = mod.expect()
            x, r = A.solve(b, params=_params(eg.MIXED))
            assert r["precision_used"] == want, (len(seen), mod.n, mod.t)
            assert r["info"] == 1 and rel(x, x_orc) < 1e-8
            mod.record(want, r)
            seen.append(want)
        # two mixed, then two FP64 probes, then the choice
        assert seen[:4] == [eg.MIXED, eg.MIXED, eg.FP64, eg.FP64]

        # an explicit FP64 request is always FP64, and it refreshes the FP64 time
        x, r = A.solve(b, params=_params(eg.FP64))
        assert r["precision_used"] == eg.FP64 and rel(x, x_orc) < 1e-8
        mod.record(eg.FP64, r)

        monkeypatch.setenv("EGPU_MIXED_AUTO", "0")
        x, r = A.solve(b, params=_params(eg.MIXED))
        assert r["precision_used"] == eg.MIXED and rel(x, x_orc) < 1e-8
        mod.record(eg.MIXED, r)
        monkeypatch.delenv("EGPU_MIXED_AUTO")

        # new values of the same operator keep the measurements
        A.update_values(v)
        want = mod.expect()
        x, r = A.solve(b, params=_params(eg.MIXED))
        assert r["precision_used"] == want and rel(x, x_orc) < 1e-8
    finally:
        A.free()


def test_caller_fp64_solves_count_and_other_methods_stay_fp64(ctx):
    p, _, _, v, b, _ = elastic_problem(meshgen.hex_cube(6))
    x_orc, _ = oracle.solve(p, v, b, method=oracle.BICGSTAB, precond=oracle.PREC_ILU0, tol=1e-8, max_iter=5000)
    A = eg.Matrix(ctx, eg.CRSPattern(p.n, p.nnz, 3, p.perm, p.rows, p.cols, p.diag), v)
    try:
        mod = Model()
        for _ in range(2):  # the caller's own FP64 solves count: no probe after the two mixed
            x, r = A.solve(b, params=_params(eg.FP64))
            assert r["precision_used"] == eg.FP64
            mod.record(eg.FP64, r)
        for _ in range(3):
            want = mod.expect()
            x, r = A.solve(b, params=_params(eg.MIXED))
            assert r["precision_used"] == want and rel(x, x_orc) < 1e-8
            mod.record(want, r)
        # GCR has no FP32 inner solver: a mixed request runs FP64 and is not timed
        x, r = A.solve(b, params=eg.SolverParams(method=eg.GCR, precond=eg.PREC_ILU0, tol=1e-8, max_iter=5000,
                                                 precision=eg.MIXED))
        assert r["precision_used"] == eg.FP64 and r["info"] == 1
        want = mod.expect()
        x, r = A.solve(b, params=_params(eg.MIXED))
        assert r["precision_used"] == want
    finally:
        A.free()
