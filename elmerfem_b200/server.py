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

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def poisson_stream(n: int, rate: float, m_lo: int, m_hi: int, seed: int, sigma: float = 1.0) -> list[Request]:
    """n requests with exponential inter-arrival times (mean 1/rate) and m log-uniform in [m_lo, m_hi]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t -= t[0]
    ms = np.floor(np.exp(rng.uniform(np.log(m_lo), np.log(m_hi + 1), size=n))).astype(int)
    ms = np.clip(ms, m_lo, m_hi)
    return [Request(i, int(ms[i]), seed * 100003 + i, float(t[i]), sigma) for i in range(n)]


class MeshPrototype:
    """Resident pattern + bound mesh of one mesh size (built once, cloned per request)."""

    def __init__(self, ctx: Context, m: int):
        self.m = m
        self.mesh = meshgen.hex_cube(m)
        self.pattern = create_matrix(self.mesh)
        self.A = Matrix(ctx, self.pattern)
        self.A.bind_assembly(self.mesh)
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
            self.protos[m] = MeshPrototype(self.ctx, m)
        return self.protos[m]

    def footprint(self, req: Request) -> float:
        return float(self.prototype(req.m).A.footprint(self.params.precond))

    def _admit(self, req: Request, now: float):
        P = self.prototype(req.m)
        A = Matrix.clone(P.A)
        rng = np.random.Generator(np.random.PCG64(req.seed))
        k = np.exp(rng.normal(0.0, req.sigma, size=P.mesh.nelem))
        load = rng.random(P.mesh.nnodes)
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
            self.prototype(r.m)
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


def run_one_at_a_time(ctx: Context, params: SolverParams, requests: list[Request], protos: dict,
                      keep_solutions: bool = False, clock=time.perf_counter) -> dict:
    """The plain drop-in path on the same stream: one egpu_iter_solve_dev at a time, arrival order."""
    import ctypes as C

    from . import _lib

    reqs = sorted(requests, key=lambda r: r.arrival)
    t0 = clock()
    for r in reqs:
        now = clock() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        P = protos[r.m]
        A = Matrix.clone(P.A)
        rng = np.random.Generator(np.random.PCG64(r.seed))
        k = np.exp(rng.normal(0.0, r.sigma, size=P.mesh.nelem))
        load = rng.random(P.mesh.nnodes)
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
