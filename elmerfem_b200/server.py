"""Continuous-batching solve server over the batched GPU solver.

Requests (a Poisson problem on a structured hex mesh of size m, with its own per-element
conductivity and nodal load) arrive over time.  The server admits them in arrival order
while their device footprint fits the HBM budget and a batch slot is free, builds each
admitted system on the device (clone of the mesh's resident pattern, GPU assembly,
Dirichlet conditions), and keeps stepping the resident batch: one FP64 refinement check
plus one chunk of FP32 inner iterations per step for every resident system.  Systems that
converge are retired (solution copied out, memory returned) and their slots reused, so
requests that arrive while others are running join the next step.

The reference has no request loop: this is the serving extension of SolveSystem
(SolverUtils.src:7531) for many independent systems.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import meshgen
from .solver import PREC_ILU0, Batch, Context, Matrix, SolverParams, create_matrix


@dataclass
class Request:
    rid: int
    m: int                   # hex mesh m^3 cells
    seed: int
    arrival: float           # seconds after the stream starts
    sigma: float = 1.0       # conductivity log-normal sigma
    admitted: float = -1.0
    finished: float = -1.0
    result: dict = field(default_factory=dict)
    x: np.ndarray | None = None
    data: tuple | None = None  # (element conductivity, nodal load), generated before the stream starts

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    def material(self, mesh) -> tuple:
        """The request's seeded element conductivity (log-normal) and nodal load, generated once.
        The serving loops generate every request's data before the stream starts, so the timed
        region measures the solvers, not the host's random-number generation."""
        if self.data is None:
            rng = np.random.Generator(np.random.PCG64(self.seed))
            k = np.exp(rng.normal(0.0, self.sigma, size=mesh.nelem))
            load = rng.random(mesh.nnodes)
            self.data = (k, load)
        return self.data


def poisson_stream(n: int, rate: float, m_lo: int, m_hi: int, seed: int, sigma: float = 1.0) -> list[Request]:
    """n requests with exponential inter-arrival times (mean 1/rate) and m log-uniform in [m_lo, m_hi]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t -= t[0]
    ms = np.floor(np.exp(rng.uniform(np.log(m_lo), np.log(m_hi + 1), size=n))).astype(int)
    ms = np.clip(ms, m_lo, m_hi)
    return [Request(i, int(ms[i]), seed * 100003 + i, float(t[i]), sigma) for i in range(n)]


def build_meshes(ms, threads: int = 0) -> dict:
    """{m: (hex mesh, CRS pattern)} for every distinct m, built on host threads (CreateMatrix
    runs in the library without the interpreter lock); a start-up cost of the serving loops."""
    import concurrent.futures as cf
    import os

    ms = sorted(set(int(m) for m in ms))

    def one(m):
        mesh = meshgen.hex_cube(m)
        return m, (mesh, create_matrix(mesh))

    nt = threads if threads > 0 else min(16, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=nt) as ex:
        return dict(ex.map(one, sorted(ms, reverse=True)))


class MeshPrototype:
    """Resident pattern + bound mesh of one mesh size (built once, cloned per request); with a
    preconditioner given, its one-time structures are built here too.  built: (mesh, pattern)
    from build_meshes, else both are made here."""

    def __init__(self, ctx: Context, m: int, precond: int | None = None, built: tuple | None = None):
        self.m = m
        if built is None:
            built = (meshgen.hex_cube(m), None)
        self.mesh = built[0]
        self.pattern = built[1] if built[1] is not None else create_matrix(self.mesh)
        self.A = Matrix(ctx, self.pattern)
        self.A.bind_assembly(self.mesh)
        if precond is not None:
            self.A.prepare(precond)
        self.con = np.sort(self.pattern.perm[self.mesh.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)


class SolveServer:
    def __init__(self, ctx: Context, params: SolverParams, hbm_budget: float = 150e9, chunk: int = 32,
                 max_resident: int = 512):
        self.ctx = ctx
        self.params = params
        self.budget = float(hbm_budget)
        self.batch = Batch(ctx, params, chunk=chunk)
        self.max_resident = max_resident
        self.protos: dict[int, MeshPrototype] = {}
        self.used = 0.0
        self.resident: dict[int, tuple[Request, Matrix, float]] = {}

    def prototype(self, m: int) -> MeshPrototype:
        if m not in self.protos:
            self.protos[m] = MeshPrototype(self.ctx, m, self.params.precond)
        return self.protos[m]

    def footprint(self, req: Request) -> float:
        return float(self.prototype(req.m).A.footprint(self.params.precond))

    def _admit(self, req: Request, now: float):
        P = self.prototype(req.m)
        A = Matrix.clone(P.A)
        k, load = req.material(P.mesh)
        req.data = None
        A.assemble_poisson(elem_k=k, load=load)
        A.dirichlet(P.con, symmetric=False)
        sid = self.batch.add_matrix(A)
        fp = self.footprint(req)
        self.used += fp
        req.admitted = now
        self.resident[sid] = (req, A, fp)

    def _retire(self, sid: int, now: float, keep_solution: bool):
        req, A, fp = self.resident.pop(sid)
        req.result = self.batch.result(sid)
        if keep_solution:
            req.x = self.batch.solution(sid)
        req.finished = now
        self.batch.remove(sid)
        A.free()
        self.used -= fp

    def run(self, requests: list[Request], keep_solutions: bool = False, clock=time.perf_counter) -> dict:
        """Serve the stream in real time; returns throughput and latency statistics."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:  # resident mesh patterns are a start-up cost (CreateMatrix once per mesh)
            r.material(self.prototype(r.m).mesh)
        queue: collections.deque[Request] = collections.deque()
        i = 0
        steps = 0
        t0 = clock()
        while i < len(reqs) or queue or self.resident:
            now = clock() - t0
            while i < len(reqs) and reqs[i].arrival <= now:
                queue.append(reqs[i])
                i += 1
            while queue and len(self.resident) < self.max_resident and \
                    self.used + self.footprint(queue[0]) <= self.budget:
                self._admit(queue.popleft(), clock() - t0)
            if self.resident:
                finished = self.batch.step()
                steps += 1
                now = clock() - t0
                for sid in finished:
                    self._retire(sid, now, keep_solutions)
            elif i < len(reqs):
                time.sleep(max(0.0, reqs[i].arrival - (clock() - t0)))
        done = [r for r in reqs if r.finished >= 0]
        lat = np.array([r.latency for r in done])
        makespan = max(r.finished for r in done) - min(r.arrival for r in done)
        return {"solves": len(done), "makespan_s": makespan, "solves_per_s": len(done) / makespan,
                "p50_ms": 1000 * float(np.percentile(lat, 50)), "p99_ms": 1000 * float(np.percentile(lat, 99)),
                "steps": steps, "converged": sum(1 for r in done if r.result.get("info") == 1)}


class NativeSolveServer:
    """The library's own continuous-batching server (egpu_server_*): admission, batch stepping
    and retirement run on a native worker thread; this class registers mesh patterns, submits
    requests and collects results."""

    def __init__(self, device: int, params: SolverParams, hbm_budget: float = 150e9, chunk: int = 32,
                 max_resident: int = 512):
        import ctypes as C

        from . import _lib
        self._C, self._lib = C, _lib
        self.params = params
        self._prm = params.to_c()
        h = C.c_void_p()
        rc = _lib.lib().egpu_server_create(device, C.byref(self._prm), float(hbm_budget), chunk, max_resident,
                                           C.byref(h))
        if rc:
            raise _lib.LibError(f"egpu_server_create: {_lib.ERRORS.get(rc, rc)}")
        self._h = h
        self.patterns: dict[int, tuple] = {}  # m -> (pattern id, (mesh, CRS pattern, Dirichlet rows))

    def _check(self, rc, what):
        if rc < 0:
            raise self._lib.LibError(f"{what}: {self._lib.ERRORS.get(rc, rc)}")
        return rc

    def pattern(self, pat) -> int:
        C = self._C
        pid = C.c_int()
        self._check(self._lib.lib().egpu_server_pattern(self._h, pat.n, pat.rows, pat.cols, pat.diag, C.byref(pid)),
                    "egpu_server_pattern")
        return pid.value

    def mesh_prototype(self, m: int, built: tuple | None = None) -> int:
        """Pattern of the m^3 hex mesh with the mesh bound for device assembly (once per m);
        built: (mesh, pattern) from build_meshes."""
        if m in self.patterns:
            return self.patterns[m][0]
        mesh, pat = built if built is not None else (meshgen.hex_cube(m), None)
        if pat is None:
            pat = create_matrix(mesh)
        pid = self.pattern(pat)
        self._check(self._lib.lib().egpu_server_pattern_mesh(
            self._h, pid, mesh.nnodes, np.ascontiguousarray(mesh.coords, np.float64), 3, mesh.nelem,
            mesh.elem_code, np.ascontiguousarray(mesh.elements, np.int32), pat.perm, pat.dofs),
            "egpu_server_pattern_mesh")
        con = np.sort(pat.perm[mesh.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)
        self.patterns[m] = (pid, (mesh, pat, con))
        return pid

    def submit(self, pid: int, values, rhs) -> int:
        C = self._C
        rid = C.c_longlong()
        self._check(self._lib.lib().egpu_server_submit(self._h, pid, np.ascontiguousarray(values, np.float64),
                                                       np.ascontiguousarray(rhs, np.float64), C.byref(rid)),
                    "egpu_server_submit")
        return rid.value

    def submit_poisson(self, pid: int, elem_k=None, nodal_k=None, load=None, con=None, symmetric=False) -> int:
        C = self._C
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (elem_k, nodal_k, load)]
        c = np.ascontiguousarray(con if con is not None else [], np.int32)
        rid = C.c_longlong()
        self._check(self._lib.lib().egpu_server_submit_poisson(
            self._h, pid, *[None if a is None else a.ctypes.data for a in arrs], c.size,
            c.ctypes.data if c.size else None, int(symmetric), C.byref(rid)), "egpu_server_submit_poisson")
        return rid.value

    def poll(self, rid: int, n: int | None = None):
        """(x, result) when the request has finished (x None when n is None), else None."""
        C = self._C
        res = self._lib.Result()
        x = None if n is None else np.zeros(n)
        rc = self._check(self._lib.lib().egpu_server_poll(self._h, rid, None if x is None else x.ctypes.data,
                                                          C.byref(res)), "egpu_server_poll")
        return (x, res.as_dict()) if rc == 1 else None

    def wait(self, rid: int, n: int | None = None, timeout: float = 600.0):
        C = self._C
        res = self._lib.Result()
        x = None if n is None else np.zeros(n)
        self._check(self._lib.lib().egpu_server_wait(self._h, rid, float(timeout),
                                                     None if x is None else x.ctypes.data, C.byref(res)),
                    "egpu_server_wait")
        return x, res.as_dict()

    def info(self) -> dict:
        st = self._lib.ServerStats()
        self._check(self._lib.lib().egpu_server_info(self._h, self._C.byref(st)), "egpu_server_info")
        return st.as_dict()

    def close(self):
        if self._h:
            self._lib.lib().egpu_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, requests: list[Request], keep_solutions: bool = False, clock=time.perf_counter) -> dict:
        """Submit the stream at its arrival times (device assembly per request) and wait for
        every result; a request's latency runs from its arrival to the server's completion."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            self.mesh_prototype(r.m)
            r.material(self.patterns[r.m][1][0])
        ids = []
        w0 = self.info()
        t0 = clock()
        for r in reqs:
            now = clock() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            pid, (mesh, pat, con) = self.patterns[r.m]
            k, load = r.material(mesh)
            r.admitted = clock() - t0
            ids.append(self.submit_poisson(pid, elem_k=k, load=load, con=con))
            r.data = None
        for r, rid in zip(reqs, ids):
            n = self.patterns[r.m][1][1].n
            x, res = self.wait(rid, n if keep_solutions else None)
            r.result = res
            r.x = x
            r.finished = r.admitted + res["seconds"]
        lat = np.array([r.latency for r in reqs])
        makespan = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
        w1 = self.info()
        info = collections.Counter(int(r.result.get("info", 0)) for r in reqs)
        return {"solves": len(reqs), "makespan_s": makespan, "solves_per_s": len(reqs) / makespan,
                "p50_ms": 1000 * float(np.percentile(lat, 50)), "p99_ms": 1000 * float(np.percentile(lat, 99)),
                "steps": w1["steps"], "converged": info.get(1, 0),
                "status_counts": {str(k): v for k, v in sorted(info.items())},
                "worker_seconds": {k: round(w1[k] - w0[k], 4) for k in ("seconds_prepare", "seconds_step",
                                                                        "seconds_retire")},
                "kernel_launches": int(w1["kernel_launches"] - w0["kernel_launches"]),
                "requeues": int(w1["requeues"] - w0["requeues"]),
                "bytes_h2d": w1["bytes_h2d"] - w0["bytes_h2d"], "bytes_d2h": w1["bytes_d2h"] - w0["bytes_d2h"]}


def run_one_at_a_time(ctx: Context, params: SolverParams, requests: list[Request], protos: dict,
                      keep_solutions: bool = False, clock=time.perf_counter) -> dict:
    """The plain drop-in path on the same stream: one egpu_iter_solve_dev at a time, arrival order."""
    import ctypes as C

    from . import _lib

    reqs = sorted(requests, key=lambda r: r.arrival)
    for r in reqs:
        r.material(protos[r.m].mesh)
    t0 = clock()
    for r in reqs:
        now = clock() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        P = protos[r.m]
        A = Matrix.clone(P.A)
        k, load = r.material(P.mesh)
        r.data = None
        A.assemble_poisson(elem_k=k, load=load)
        A.dirichlet(P.con, symmetric=False)
        x = np.zeros(A.n)
        res = _lib.Result()
        prm = params.to_c()
        rc = _lib.lib().egpu_iter_solve(A.handle, A.rhs(), x, C.byref(prm), C.byref(res))
        r.result = res.as_dict()
        r.result["info"] = rc
        if keep_solutions:
            r.x = x
        r.finished = clock() - t0
        A.free()
    lat = np.array([r.latency for r in reqs])
    makespan = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
    return {"solves": len(reqs), "makespan_s": makespan, "solves_per_s": len(reqs) / makespan,
            "p50_ms": 1000 * float(np.percentile(lat, 50)), "p99_ms": 1000 * float(np.percentile(lat, 99)),
            "converged": sum(1 for r in reqs if r.result.get("info") == 1)}
