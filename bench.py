"""Benchmark of the B200 linear-system path (solves/s), one JSON line on rank 0.

Headline workload (default): steady 3D Poisson on the unit cube, structured 128^3 trilinear
hexahedra (2,146,689 DOFs, 57.07M nonzeros), per-element conductivity k ~ logN(0, 1) (seed 1),
nodal source sin(pi x) sin(pi y) sin(pi z), zero Dirichlet on all faces with symmetric
elimination, CG + Diagonal preconditioning, tolerance 1e-10 on ||Ax-b||/||b|| of the scaled
system.  A step is one SolveLinearSystem of the assembled system (scaling, preconditioner,
Krylov loop, back-scaling) with the mixed FP32-inner / FP64-refinement solver; the FP64 drop-in
solver is timed on the same system in the same run, and both solutions are compared with one
full FP64 solve of the oracle (the CPU restatement of the reference path), whose time is the
CPU baseline.  The same line carries two nested sections measured in the same run:
  "batched"  512 independent tet Poisson systems (m log-uniform in [8, 60]) in one persistent
             mixed-precision launch, against the FP64 drop-in one system at a time;
  "serving"  a 200/s Poisson-process stream of hex Poisson requests (m log-uniform in
             [16, 128]) through the native continuous-batching server, against the FP64
             drop-in one request at a time on the same stream.
Inputs are synthetic (seeded; no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

Workloads: poisson128_cg_jacobi (default), poisson96_cg_jacobi, poisson32_bicgstab_ilu0,
elastic64_bicgstab_ilu0 (single systems: mixed solve timed, FP64 drop-in beside it), batch512_tet_cg_jacobi,
serve_hex_bicgstab_ilu0 (the nested sections as lines of their own).  --no-nested drops the
nested sections.

--impl reference times the oracle on the host cores on the same workload: every step is one
complete FP64 solve (SpMV and vector operations on every host thread).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s, p50/p99 latency: mixed vs FP64 GPU at 1e-8 rel err; SpMV GB/s"
UNIT = "solves/s"


# ------------------------------------------------------------------------------------- workloads
def workload_spec(name):
    from elmerfem_b200 import meshgen

    if name == "poisson128_cg_jacobi":
        def build():
            m = meshgen.hex_cube(128)
            return dict(mesh=m, elem_k=meshgen.lognormal_conductivity(m.nelem, 1.0, 1),
                        load=meshgen.sine_source(m.coords), bc=range(1, 7), symmetric=True)
        return build, dict(method=1, precond=1, tol=1e-10, max_iter=20000), \
            {"workload": "poisson_hex128_lognormal_cg_jacobi", "mesh": "128^3 hex 808", "dofs": 2146689,
             "method": "CG", "preconditioner": "Diagonal", "tol": 1e-10}
    if name == "poisson96_cg_jacobi":
        # profiling-size variant of the 128^3 workload (matrix 146 MB in FP32: still larger than L2)
        def build():
            m = meshgen.hex_cube(96)
            return dict(mesh=m, elem_k=meshgen.lognormal_conductivity(m.nelem, 1.0, 1),
                        load=meshgen.sine_source(m.coords), bc=range(1, 7), symmetric=True)
        return build, dict(method=1, precond=1, tol=1e-10, max_iter=20000), \
            {"workload": "poisson_hex96_lognormal_cg_jacobi", "mesh": "96^3 hex 808", "dofs": 912673,
             "method": "CG", "preconditioner": "Diagonal", "tol": 1e-10}
    if name == "elastic64_bicgstab_ilu0":
        def build():
            m = meshgen.hex_cube(64)
            return dict(mesh=m, elastic=True, bc=[1], symmetric=False)
        return build, dict(method=2, precond=2, tol=1e-8, max_iter=20000), \
            {"workload": "elasticity_hex64_bicgstab_ilu0", "mesh": "64^3 hex 808, 3 DOFs/node", "dofs": 823875,
             "method": "BiCGStab", "preconditioner": "ILU0", "tol": 1e-8, "E": 200e9, "nu": 0.3,
             "body_force": [0, 0, -1e4]}
    if name == "poisson32_bicgstab_ilu0":
        def build():
            m = meshgen.hex_cube(32)
            return dict(mesh=m, elem_k=None, load=np.ones(m.nnodes), bc=range(1, 7), symmetric=False)
        return build, dict(method=2, precond=2, tol=1e-10, max_iter=1000), \
            {"workload": "poisson_hex32_bicgstab_ilu0", "mesh": "32^3 hex 808", "dofs": 35937,
             "method": "BiCGStab", "preconditioner": "ILU0", "tol": 1e-10}
    raise SystemExit(f"unknown workload {name}")


def compact_offset_fraction(pat):
    """Share of SELL-32 entries whose column offsets the library stores per entry: a slice of
    32 existing rows with one common offset list (col - row) stores it once (the compact
    layout of egpu_matrix_bind), every other slice one 2-byte offset per entry."""
    n = pat.n
    rows = np.asarray(pat.rows, np.int64) - 1
    cols = np.asarray(pat.cols, np.int64) - 1
    lens = np.diff(rows)
    row_of = np.repeat(np.arange(n, dtype=np.int64), lens)
    k = np.arange(rows[-1], dtype=np.int64) - np.repeat(rows[:-1], lens)
    off = cols - row_of + (1 << 20)
    h1 = np.zeros(n, np.uint64)
    h2 = np.zeros(n, np.uint64)
    np.add.at(h1, row_of, (off * (k * 2654435761 + 97)).astype(np.uint64))
    np.add.at(h2, row_of, ((off * 40503 + k) * (off ^ 0x5bd1e995)).astype(np.uint64))
    ns = (n + 31) // 32
    full = ns if n % 32 == 0 else ns - 1
    wmax = np.zeros(ns, np.int64)
    np.maximum.at(wmax, np.arange(n) // 32, lens)
    tot = 32 * wmax.sum()
    lf, a1, a2 = lens[:32 * full].reshape(full, 32), h1[:32 * full].reshape(full, 32), h2[:32 * full].reshape(full, 32)
    shared = (lf == lf[:, :1]).all(1) & (a1 == a1[:, :1]).all(1) & (a2 == a2[:, :1]).all(1) & (lf[:, 0] > 0)
    return 1.0 - float((32 * wmax[:full][shared]).sum()) / float(tot)


def algorithmic_bytes_per_iter(method, precond, precision, n, nnz, cols16, off_frac=1.0, unit_diag=False, sweeps=0):
    """Bytes one Krylov iteration must move (matrix streamed once per SpMV pass, vectors once).

    CG+Diagonal, FP32 inner (refinement): SpMV 4z values + 2z·off_frac offsets (int16 column
    offsets, stored once per slice where all rows share them) or 4z cols + 4n rowptr + P gather
    4n + Q write 4n + epilogue P 4n; P update 12n; x/r/z update 32n.  When the scaled diagonal
    is 1.0f everywhere (unit_diag) the Jacobi step is the identity: no diagonal read and no Z
    write, 48n of vectors instead of 60n.
    CG+Diagonal, FP64 drop-in (x_k residual fused in the next SpMV): SpMV 8z + the same offsets
    + 4n + 16n gathers + 8n write + 16n epilogue; P update 24n; update 64n.
    """
    cbytes = (2 * off_frac if cols16 else 4) * nnz
    if method == 1 and precond in (0, 1):
        if precision == "mixed":
            return 4 * nnz + cbytes + (48 if (unit_diag or precond == 0) else 60) * n
        return 8 * nnz + cbytes + 132 * n
    # BiCGStab: two SpMV passes (+x fused in FP64) and two preconditioner applications
    if precision == "mixed":
        m = 4 * nnz + cbytes
        tri = (8 * nnz + 16 * n) if precond == 2 else 0
        if precond == 2 and sweeps > 0:
            # per application: `sweeps` passes over each triangle's half of the factor entries
            # (values and offsets), each gathering its input and reading / writing 12n of
            # vectors, the inverted diagonal (4n) in the upper sweeps, and z0 (4n) once
            tri = 2 * (2 * sweeps * ((4 * nnz + cbytes) / 2 + 12 * n) + sweeps * 4 * n + 4 * n)
        return 2 * m + tri + 120 * n
    m = 8 * nnz + cbytes
    tri = (12 * nnz + 32 * n) if precond == 2 else 0
    return 2 * m + tri + 260 * n


# ------------------------------------------------------------------------------------- clocks
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------- helpers
def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if os.environ.get("BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def _coll_device(pg, device):
    # gloo reduces host tensors, NCCL device tensors
    if pg is not None and pg.get_backend() == "gloo":
        return "cpu"
    return device if device is not None else "cuda"


def reduce_max(pg, value, device):
    """Max over ranks (every timed number of a multi-GPU run is the slowest rank's)."""
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=_coll_device(pg, device))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    if pg is not None:
        import torch

        pg.all_reduce(torch.zeros(1, device=_coll_device(pg, device)))


def read_peaks():
    try:
        pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def read_traffic(workload):
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        return t.get(workload)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------------------------------------- CPU arm
def oracle_mod():
    """The oracle, built for this host (-march=native) before its first use."""
    import oracle

    if oracle._lib is None:
        oracle.use_native()
    return oracle


def host_threads():
    return os.cpu_count() or 1


def l2_note(n, nnz):
    """Working sets below twice the 126 MB L2 run from L2 between solves unless flushed."""
    ws = 12 * nnz + 80 * n
    small = ws < 2 * 126 * 2**20
    return small, (f"working set {ws / 2**20:.0f} MB < 2x L2: 256 MB L2 flush before every timed step, "
                   "per-step CUDA events" if small else
                   f"working set {ws / 2**20:.0f} MB larger than L2; no flush needed")


def headline_config(cfg, n, nnz, world):
    """config of the single-system lines, identical in both arms"""
    return dict(cfg, parallelism=f"replicas{world}", l2=l2_note(n, nnz)[1])


def oracle_system(w):
    """(pattern, Values, RHS) of a single-system workload, assembled by the oracle."""
    oracle = oracle_mod()

    m = w["mesh"]
    if w.get("elastic"):
        p = oracle.create_pattern(m, dofs=3)
        vals, rhs = oracle.assemble_elastic(m, p, 200e9, 0.3, (0.0, 0.0, -1e4))
        nodes = p.perm[m.boundary_nodes(w["bc"]) - 1]
        con = np.sort(np.concatenate([3 * (nodes - 1) + d for d in (1, 2, 3)])).astype(np.int32)
    else:
        p = oracle.create_pattern(m)
        nodal_k = None if w["elem_k"] is not None else np.ones(m.nnodes)
        vals, rhs = oracle.assemble_poisson(m, p, elem_k=w["elem_k"], nodal_k=nodal_k, load=w["load"])
        con = np.sort(p.perm[m.boundary_nodes(w["bc"]) - 1]).astype(np.int32)
    oracle.dirichlet(p, vals, rhs, con, symmetric=w["symmetric"])
    return p, vals, rhs


def oracle_solve_timed(p, values, rhs, method, precond, tol, threads, max_iter=20000):
    """One complete FP64 solve of the oracle (scaling, preconditioner, Krylov loop,
    back-scaling) with its SpMV and vector operations on `threads` host threads; the ILU
    triangular solves stay sequential, as in the reference.  Returns (x, result dict)."""
    oracle = oracle_mod()

    return oracle.solve(p, values, rhs, method=method, precond=precond, max_iter=max_iter, tol=tol,
                        threads=threads, blas_threads=threads)


def reference_systems_rate(kind, tol, systems, requests, rate, target_s, start=0):
    """CPU reference of the batched / serving workloads: the oracle solves the workload's own
    systems one at a time in FP64 (the reference's only mode) in their seeded order, on every
    host thread, until about target_s seconds of solve time; returns (systems per second,
    systems solved, solve seconds, config).  Sizes are drawn independently, so the prefix is a
    random sample of the mix.  Assembly and Dirichlet rows are set up outside the timing, as in
    the GPU arms."""
    oracle = oracle_mod()
    from elmerfem_b200 import meshgen, server

    threads = host_threads()
    if kind == "batched":
        ms = batch_sizes(systems)
        method, prec = oracle.CG, oracle.PREC_DIAGONAL

        def system(i):
            mesh = meshgen.tet_cube(int(ms[i]))
            p = oracle.create_pattern(mesh)
            k = meshgen.lognormal_conductivity(mesh.nelem, 0.5, 1000 + i)
            vals, rhs = oracle.assemble_poisson(mesh, p, elem_k=k, load=np.zeros(mesh.nnodes))
            con = np.sort(p.perm[mesh.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)
            oracle.dirichlet(p, vals, rhs, con, symmetric=True)
            b = batch_rhs(i, p.n, con)
            return p, vals, b
        count = systems
    else:
        reqs = server.poisson_stream(requests, rate=rate, m_lo=16, m_hi=128, seed=1, sigma=1.0)
        method, prec = oracle.BICGSTAB, oracle.PREC_ILU0

        def system(i):
            r = reqs[i]
            mesh = meshgen.hex_cube(r.m)
            p = oracle.create_pattern(mesh)
            k, load = r.material(mesh)
            r.data = None
            vals, rhs = oracle.assemble_poisson(mesh, p, elem_k=k, load=load)
            con = np.sort(p.perm[mesh.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)
            oracle.dirichlet(p, vals, rhs, con, symmetric=False)
            return p, vals, rhs
        count = len(reqs)
    t, n = 0.0, 0
    while t < target_s and n < count:
        p, vals, b = system((start + n) % count)
        _, r = oracle_solve_timed(p, vals, b, method, prec, tol, threads)
        t += r["seconds"]
        n += 1
    return n / t, n, t, threads


def run_reference_systems(args, world):
    """Reference arm of the batched and serving workloads (their own lines)."""
    kind = "batched" if args.workload == "batch512_tet_cg_jacobi" else "serving"
    target = 8.0 if kind == "batched" else 20.0
    for _ in range(args.warmup):
        reference_systems_rate(kind, args.tol, args.systems, args.requests, args.rate, min(2.0, target))
    rates, n, t = [], 0, 0.0
    for _ in range(args.steps):
        r, n, t, threads = reference_systems_rate(kind, args.tol, args.systems, args.requests, args.rate, target)
        rates.append(r)
    value = statistics.median(rates)
    cfg = batch_config(args, world) if kind == "batched" else serve_config(args, world, "native (egpu_server_*)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"per step: the first {n} systems in seeded order, whole FP64 oracle solves "
                                       f"({t:.1f} s of solve time), solved one at a time"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args, rank, world, pg):
    """Reference arm: every step is one complete FP64 oracle solve of the workload's system
    (its time is the step's time), after W untimed ones."""
    if rank != 0:
        return
    if args.workload in ("batch512_tet_cg_jacobi", "serve_hex_bicgstab_ilu0"):
        return run_reference_systems(args, world)
    build, solve_kw, cfg = workload_spec(args.workload)
    p, vals, rhs = oracle_system(build())
    threads = host_threads()

    def step():
        _, r = oracle_solve_timed(p, vals, rhs, solve_kw["method"], solve_kw["precond"], solve_kw["tol"], threads,
                                  solve_kw["max_iter"])
        return r

    for _ in range(args.warmup):
        step()
    res = [step() for _ in range(args.steps)]
    times = [r["seconds"] for r in res]
    med = statistics.median(times)
    value = 1.0 / med
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * med, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(cfg, p.n, p.nnz, world),
            "iterations": {"fp64": res[-1]["iters"]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"every step one complete FP64 oracle solve ({res[-1]['iters']} iterations, "
                                       f"median {med:.2f} s); SpMV and vector operations on {threads} threads, "
                                       "ILU triangular solves sequential as in the reference"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------- GPU arm
def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_gpu(args, rank, world, local, pg):
    import torch

    import elmerfem_b200 as eg

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = eg.Context(local)
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    build, solve_kw, cfg = workload_spec(args.workload)
    w = build()
    m = w["mesh"]
    dofs = 3 if w.get("elastic") else 1
    pat = eg.create_matrix(m, dofs=dofs)
    A = eg.Matrix(ctx, pat)
    A.bind_assembly(m)
    if w.get("elastic"):
        A.assemble_elastic(200e9, 0.3, (0.0, 0.0, -1e4))
        nodes = pat.perm[m.boundary_nodes(w["bc"]) - 1]
        con = np.sort(np.concatenate([3 * (nodes - 1) + d for d in (1, 2, 3)])).astype(np.int32)
    else:
        nodal_k = None if w["elem_k"] is not None else np.ones(m.nnodes)
        A.assemble_poisson(elem_k=w["elem_k"], nodal_k=nodal_k, load=w["load"])
        con = np.sort(pat.perm[m.boundary_nodes(w["bc"]) - 1]).astype(np.int32)
    A.dirichlet(con, symmetric=w["symmetric"])
    n, nnz = pat.n, pat.nnz
    cols16 = True  # every structured workload here has |col-row| < 32768
    mixed = eg.SolverParams(method=solve_kw["method"], precond=solve_kw["precond"], tol=solve_kw["tol"],
                            max_iter=solve_kw["max_iter"], precision=eg.MIXED, inner_tol=args.inner_tol)
    fp64 = eg.SolverParams(method=solve_kw["method"], precond=solve_kw["precond"], tol=solve_kw["tol"],
                           max_iter=solve_kw["max_iter"])
    x = torch.zeros(n, dtype=torch.float64, device=dev)

    def step(prm):
        with torch.cuda.stream(ext):
            x.zero_()
        return A.solve_dev(None, x.data_ptr(), prm)

    # warm-up: two FP64 drop-in solves, then the mixed requests.  The library measures both
    # paths on the matrix (each path's first solve carries one-time set-up) and, from the third
    # mixed request on, runs the faster one; the second mixed request is always on the mixed
    # path and its solution is kept for the error figures, as is the FP64 drop-in's.
    for _ in range(2):
        r64 = step(fp64)
    x64 = x.cpu().numpy()
    for i in range(max(2, args.warmup)):
        r = step(mixed)
        if i == 1:
            rm, xm = r, x.cpu().numpy()
    assert rm["precision_used"] == eg.MIXED

    small, note = l2_note(n, nnz)
    flush_buf = torch.empty(64 * 2**20, dtype=torch.float32, device=dev) if small else None

    def timed(fn, k):
        """k calls of fn on the solver's stream: (device seconds, results)"""
        out = []
        if not small:
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(ext)
            for _ in range(k):
                out.append(fn())
            a1.record(ext)
            torch.cuda.synchronize()
            return a0.elapsed_time(a1) / 1000.0, out
        ev = []
        for _ in range(k):
            with torch.cuda.stream(ext):
                flush_buf.fill_(float(len(ev)))
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(ext)
            out.append(fn())
            a1.record(ext)
            ev.append((a0, a1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / 1000.0, out

    # ---- timed: mixed, device-resident inputs
    launches0 = ctx.kernel_launches
    barrier(pg, dev)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t, results = timed(lambda: step(mixed), args.steps)
    barrier(pg, dev)
    launches = ctx.kernel_launches - launches0
    t = reduce_max(pg, t, dev)
    value = world * args.steps / t
    lat = sorted(r["seconds"] for r in results)

    # ---- roofline of the dominant kernel: the persistent Krylov kernel of the path the timed
    # requests took (FP32 inner for mixed, FP64 for the drop-in)
    n_mixed_path = sum(1 for r in results if r.get("precision_used") == eg.MIXED)
    path = "mixed" if 2 * n_mixed_path >= len(results) else "fp64"
    on_path = [r for r in results if (r.get("precision_used") == eg.MIXED) == (path == "mixed")]
    iters = sum(r["iters"] for r in on_path)
    sec_k = sum(r["seconds_krylov"] for r in on_path)
    nlaunch = sum(r["krylov_launches"] for r in on_path)
    off_frac = compact_offset_fraction(pat)
    # the library's FP32 inner CG drops the Jacobi step when the scaled diagonal rounds to 1.0f
    # everywhere (as it does after the symmetric scaling of a positive diagonal)
    unit_diag = False
    if solve_kw["precond"] == eg.PREC_DIAGONAL:
        dv = A.values()[pat.diag - 1]
        dsc = 1.0 / np.sqrt(np.abs(dv))
        unit_diag = bool(np.all((dv * dsc * dsc).astype(np.float32) == np.float32(1.0)))
    sweeps = max((r.get("ilu_sweeps_used", 0) for r in on_path), default=0)
    bpi = algorithmic_bytes_per_iter(solve_kw["method"], solve_kw["precond"], path, n, nnz, cols16, off_frac,
                                     unit_diag, sweeps)
    peak, peak_kind = read_peaks()
    achieved = bpi * iters / sec_k / 1e9
    traffic = read_traffic(cfg["workload"])
    ty, what = ("float", "FP32 inner") if path == "mixed" else ("double", "FP64 drop-in")
    if solve_kw["method"] == eg.CG:
        kernel_name = f"cg_kernel<{ty},LPR,int16 cols> (persistent {what} CG)"
    else:
        ilu_what = (f"ILU0 by {sweeps} Jacobi sweeps per triangle in the kernel)" if sweeps else
                    "ILU0 triangular solves in the kernel)")
        kernel_name = (f"bicgstab_kernel<{ty},LPR,int16 cols> (persistent {what} BiCGStab, "
                       + (ilu_what if solve_kw["precond"] == eg.PREC_ILU0 else "no ILU)"))

    # ---- FP64 drop-in on the same system
    t64 = []
    for _ in range(args.fp64_steps):
        torch.cuda.synchronize()
        dt, (rr,) = timed(lambda: step(fp64), 1)
        t64.append(dt)
    fp64_rate = 1.0 / statistics.median(t64)
    bpi64 = algorithmic_bytes_per_iter(solve_kw["method"], solve_kw["precond"], "fp64", n, nnz, cols16, off_frac)
    ach64 = bpi64 * rr["iters"] / rr["seconds_krylov"] / 1e9

    # ---- end to end through the public C ABI with host buffers (pinned)
    b_host = torch.from_numpy(A.rhs()).pin_memory()
    x_host = torch.zeros(n, dtype=torch.float64).pin_memory()
    import ctypes as C

    from elmerfem_b200 import _lib

    def step_host():
        x_host.zero_()
        prm = mixed.to_c()
        res = _lib.Result()
        bp = np.ctypeslib.as_array(C.cast(b_host.data_ptr(), C.POINTER(C.c_double)), shape=(n,))
        xp = np.ctypeslib.as_array(C.cast(x_host.data_ptr(), C.POINTER(C.c_double)), shape=(n,))
        rc = _lib.lib().egpu_iter_solve(A.handle, bp, xp, C.byref(prm), C.byref(res))
        assert rc == 1, rc
        return float(xp[0])

    step_host()
    barrier(pg, dev)
    torch.cuda.synchronize()
    te, _ = timed(step_host, args.steps)
    te = reduce_max(pg, te, dev)
    e2e = world * args.steps / te

    # ---- element assembly (not part of the step): device time of one egpu_assemble_poisson
    # (element conductivity upload, zeroing, the colour launches), per element.  Estimated work
    # per 8-node element (2x2x2 Gauss points): Jacobian 72 FMA, its inverse ~40 FLOP,
    # dN/dx 72 FMA, the 8x8 stiffness 192 FMA and the load 8 FMA per point, about 5.6 kFLOP;
    # bytes: 8 nodes x (24 B coordinates + 4 B index), the element's k, 64 slot indices and
    # read-modify-writes of 64 values and 8 right-hand-side entries (1,640 B).
    assembly = None
    if not w.get("elastic") and m.elem_code == 808:
        ta = []
        for _ in range(3):
            torch.cuda.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(ext)
            A.assemble_poisson(elem_k=w["elem_k"], nodal_k=nodal_k, load=w["load"])
            a1.record(ext)
            torch.cuda.synchronize()
            ta.append(a0.elapsed_time(a1) / 1000.0)
            A.dirichlet(con, symmetric=w["symmetric"])
        t_as = statistics.median(ta)
        ne = m.nelem
        assembly = {"ms": 1000 * t_as, "elements": ne, "elements_per_s": ne / t_as,
                    "gflops_fp64_est": 5600.0 * ne / t_as / 1e9, "gbs_est": 1640.0 * ne / t_as / 1e9,
                    "hbm_frac_est": 1640.0 * ne / t_as / 1e9 / peak}

    # ---- the oracle: one complete FP64 solve of the same system on the host cores (rank 0,
    # N = 1): the CPU baseline, and the reference solution both GPU results are measured against
    cpu, err_oracle = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        oracle = oracle_mod()

        op = oracle.Pattern(n, nnz, dofs, pat.perm, pat.rows, pat.cols, pat.diag, 0, 0, 0, 0)
        threads = host_threads()
        x_orc, ro = oracle_solve_timed(op, A.values(), A.rhs(), solve_kw["method"], solve_kw["precond"],
                                       solve_kw["tol"], threads, solve_kw["max_iter"])
        cpu = {"value": 1.0 / ro["seconds"], "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"one complete FP64 oracle solve ({ro['iters']} iterations, {ro['seconds']:.2f} s); "
                         f"SpMV and vector operations on {threads} threads, ILU triangular solves sequential "
                         "as in the reference"}
        err_oracle = {"mixed": rel(xm, x_orc), "fp64": rel(x64, x_orc), "oracle_iters": ro["iters"],
                      "oracle_info": ro["info"], "bound": 1e-8}

    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * t / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 inner / f64 refinement" if path == "mixed" else "f64", "data": "synthetic",
                "config": headline_config(cfg, n, nnz, world),
                "latency_ms": {"p50": 1000 * lat[len(lat) // 2], "p99": 1000 * lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
                "iterations": {"mixed_inner_total": rm["iters"], "refinements": rm["refinements"],
                               "fp64": r64["iters"]},
                # a mixed request runs the FP64 drop-in on values it was measured faster on
                "path_of_timed_steps": {"mixed": sum(1 for r in results if r.get("precision_used") == 1),
                                        "fp64": sum(1 for r in results if r.get("precision_used") == 0),
                                        "ilu_sweeps": sweeps},
                "fp64": {"solves_per_s": fp64_rate, "ms_per_solve": 1000 * statistics.median(t64),
                         "krylov_gbs": ach64},
                "speedup_mixed_vs_fp64": value / world / fp64_rate,
                "rel_err_vs_oracle": err_oracle,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": kernel_name,
                             "bytes_per_iter": bpi, "launches": nlaunch,
                             "per_entry_offset_share": off_frac, "unit_diagonal": unit_diag},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8 * n},
                "gpu_launches": launches,
                "clocks": clk.summary(),
                "cpu_baseline": cpu,
                "assembly": assembly}
    A.free()
    del x, flush_buf, b_host, x_host
    torch.cuda.synchronize()
    ctx.close()
    if args.workload == "poisson128_cg_jacobi" and not args.no_nested:
        bat = section_batched(args, rank, world, local, pg, nested=True)
        srv = section_serving(args, rank, world, local, pg, nested=True)
        if line is not None:
            line["batched"], line["serving"] = bat, srv
    if line is not None:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------- batch (C4)
def batch_sizes(nsys):
    rng = np.random.Generator(np.random.PCG64(1))
    return np.clip(np.floor(np.exp(rng.uniform(np.log(8), np.log(61), size=nsys))).astype(int), 8, 60)


def batch_rhs(i, n, con):
    b = np.random.Generator(np.random.PCG64(5000 + i)).random(n)
    b[con - 1] = 0.0
    return b


def batch_config(args, world):
    return {"workload": "batched_tet_poisson_512_cg_jacobi", "systems": int(args.systems), "m_range": [8, 60],
            "method": "CG", "preconditioner": "Diagonal", "tol": args.tol, "parallelism": f"replicas{world}",
            "l2": "working set larger than L2"}


def section_batched(args, rank, world, local, pg, nested=False):
    """512 independent tet Poisson systems (m log-uniform in [8, 60]) in one batched mixed solve
    per step, against the FP64 drop-in one system at a time; returns the section's dict."""
    import torch

    import elmerfem_b200 as eg
    from elmerfem_b200 import meshgen

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = eg.Context(local)
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    nsys = args.systems
    ms = batch_sizes(nsys)
    protos, mats, bs, cons = {}, [], [], []
    for i, m in enumerate(ms):
        if m not in protos:
            mesh = meshgen.tet_cube(int(m))
            pat = eg.create_matrix(mesh)
            P = eg.Matrix(ctx, pat)
            P.bind_assembly(mesh)
            con = np.sort(pat.perm[mesh.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)
            protos[m] = (mesh, P, con)
        mesh, P, con = protos[m]
        A = eg.Matrix.clone(P)
        k = meshgen.lognormal_conductivity(mesh.nelem, 0.5, 1000 + i)
        A.assemble_poisson(elem_k=k, load=None)
        A.dirichlet(con, symmetric=True)
        mats.append(A)
        cons.append(con)
        bs.append(torch.from_numpy(batch_rhs(i, A.n, con)).to(dev))
    torch.cuda.synchronize()
    ndofs = int(sum(A.n for A in mats))
    nnz = int(sum(A.nnz for A in mats))
    prm = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=args.tol, max_iter=20000,
                          inner_tol=args.inner_tol)
    steps = args.batch_steps if nested else args.steps
    warmup = 2 if nested else args.warmup
    tuned = {}

    def batch_step(tune=False):
        B = eg.Batch(ctx, prm, chunk=args.chunk)
        ids = [B.add_matrix(A, b.data_ptr()) for A, b in zip(mats, bs)]
        if tune:  # autotuner on the first warm-up batch; the timed batches reuse its choice
            tuned.update(B.tune())
        elif tuned:
            B.set_config(tuned)
        B.solve()
        res = [B.result(i) for i in ids]
        return B, ids, res

    for wu in range(warmup):
        B, _, _ = batch_step(tune=(wu == 0 and not args.no_tune))
        B.free()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ctx.kernel_launches
    barrier(pg, dev)
    torch.cuda.synchronize()
    times, kms, allres = [], [], None
    with ClockSampler(local) as clk:
        for _ in range(steps):
            e0.record(ext)
            B, ids, res = batch_step()
            e1.record(ext)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1000.0)
            kms.append(B.last_launch_ms())
            if allres is None:
                allres = res
                xs_b = [B.solution(i) for i in ids]
            B.free()
    launches = ctx.kernel_launches - launches0
    t = reduce_max(pg, sum(times), dev)
    value = world * nsys * steps / t
    # end to end: every step uploads all right-hand sides from one pinned host buffer, solves the
    # batch and reads every solution back to host memory through the public calls
    offs = np.concatenate([[0], np.cumsum([A.n for A in mats])]).astype(np.int64)
    hb = torch.empty(ndofs, dtype=torch.float64).pin_memory()
    for j, b in enumerate(bs):
        hb[offs[j]:offs[j + 1]].copy_(b.cpu())
    db = torch.empty(ndofs, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    barrier(pg, dev)
    te = []
    for _ in range(steps):
        e0.record(ext)
        with torch.cuda.stream(ext):
            db.copy_(hb, non_blocking=True)
        B = eg.Batch(ctx, prm, chunk=args.chunk)
        ids = [B.add_matrix(A, db.data_ptr() + 8 * int(offs[j])) for j, A in enumerate(mats)]
        if tuned:
            B.set_config(tuned)
        B.solve()
        xs_e = [B.solution(i) for i in ids]
        e1.record(ext)
        torch.cuda.synchronize()
        te.append(e0.elapsed_time(e1) / 1000.0)
        B.free()
    e2e_err = max(rel(xe, xb) for xe, xb in zip(xs_e, xs_b))
    t_e2e = reduce_max(pg, sum(te), dev)
    # the pinned buffer was used on the library's stream: free it while that stream exists
    del hb, db
    torch.cuda.synchronize()
    # FP64 drop-in one system at a time on the same systems
    fp = eg.SolverParams(method=eg.CG, precond=eg.PREC_DIAGONAL, tol=args.tol, max_iter=20000)
    x64 = [torch.zeros(A.n, dtype=torch.float64, device=dev) for A in mats]
    torch.cuda.synchronize()
    e0.record(ext)
    it64 = 0
    for A, b, xv in zip(mats, bs, x64):
        r = A.solve_dev(b.data_ptr(), xv.data_ptr(), fp)
        it64 += r["iters"]
    e1.record(ext)
    torch.cuda.synchronize()
    t64 = e0.elapsed_time(e1) / 1000.0
    x64h = [xv.cpu().numpy() for xv in x64]
    errs = [rel(xs_b[j], x64h[j]) for j in range(nsys)]
    peak, peak_kind = read_peaks()
    inner_iters = sum(r["iters"] for r in allres)

    # the batched CG drops the Jacobi step for systems whose scaled diagonal rounds to 1.0f
    def unit_diag_of(A):
        dv = A.values()[A.pattern.diag - 1]
        dsc = 1.0 / np.sqrt(np.abs(dv))
        return bool(np.all((dv * dsc * dsc).astype(np.float32) == np.float32(1.0)))

    units = [unit_diag_of(A) for A in mats]
    bpi = sum(algorithmic_bytes_per_iter(1, 1, "mixed", A.n, A.nnz, True, 1.0, u) * r["iters"]
              for A, r, u in zip(mats, allres, units))
    # device time of the batched launch (the team solver runs every solve in one launch; on the
    # stepwise path this is the last chunk only, and the whole step is the honest figure)
    teams = os.environ.get("EGPU_BATCH_TEAMS", "1") != "0"
    kt = float(np.mean(kms)) / 1000.0 if teams and kms and min(kms) > 0 else t / steps
    # against the FP64 oracle: a seeded sample of systems (the smallest six and two more)
    out = None
    if rank == 0:
        oracle = oracle_mod()

        order = np.argsort(ms, kind="stable")
        rng = np.random.default_rng(17)
        pick = list(order[:6]) + list(rng.choice(order[6:nsys // 2], size=2, replace=False))
        eo, e64o = [], []
        for j in pick:
            A = mats[j]
            op = oracle.Pattern(A.n, A.nnz, 1, A.pattern.perm, A.pattern.rows, A.pattern.cols, A.pattern.diag,
                                0, 0, 0, 0)
            xo, _ = oracle_solve_timed(op, A.values(), bs[j].cpu().numpy(), oracle.CG, oracle.PREC_DIAGONAL, args.tol,
                                       host_threads())
            eo.append(rel(xs_b[j], xo))
            e64o.append(rel(x64h[j], xo))
        cpu = None
        if world == 1 and not args.no_cpu:
            cr, cn, ct, cth = reference_systems_rate("batched", args.tol, nsys, 0, 0.0, args.cpu_seconds)
            cpu = {"value": cr, "unit": UNIT, "cores": cth, "kind": "port",
                   "sample": f"the first {cn} systems in seeded order, whole FP64 oracle solves one at a time "
                             f"({ct:.1f} s)"}
        out = {"value": value, "unit": UNIT, "steps": steps, "ms_per_step": 1000 * t / steps,
               "config": dict(batch_config(args, world), dofs_total=ndofs, nnz_total=nnz,
                              solver=("team (k_batch_team: one launch, a team of CTAs per system)" if teams
                                      else "stepwise (k_batch_inner chunks)"),
                              # the autotuner sets up the stepwise kernel (the first warm-up batch
                              # runs on it); the team solver sizes its teams from the systems
                              autotuned_stepwise=tuned or None),
               "dtype": "f32 inner / f64 refinement",
               "fp64_one_at_a_time": {"solves_per_s": nsys / t64, "seconds": t64, "iters_total": it64},
               "speedup_vs_fp64": value / world / (nsys / t64),
               "rel_err_vs_fp64_max": max(errs),
               "rel_err_vs_oracle": {"systems": [int(j) for j in pick], "m": [int(ms[j]) for j in pick],
                                     "mixed_max": max(eo), "fp64_max": max(e64o), "bound": 1e-8},
               "iterations": {"inner_total": inner_iters},
               "roofline": {"bound": "hbm", "achieved": bpi / kt / 1e9, "peak": peak,
                            "unit": "GB/s", "frac": bpi / kt / 1e9 / peak, "traffic": None,
                            "peak_kind": peak_kind,
                            "kernel": "k_batch_team (one cooperative launch: every system's whole mixed solve, "
                                      "FP64 residuals included)",
                            "kernel_ms": 1000 * kt,
                            "whole_step_achieved": bpi / (t / steps) / 1e9,
                            "unit_diagonal_systems": int(sum(units))},
               "e2e": {"value": world * nsys * steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * ndofs,
                       "d2h_bytes_per_step": 8 * ndofs, "max_rel_diff_vs_device_timed": e2e_err},
               "gpu_launches": launches, "clocks": clk.summary(), "cpu_baseline": cpu}
    for A in mats:
        A.free()
    for _, P, _ in protos.values():
        P.free()
    del bs, x64
    torch.cuda.synchronize()
    ctx.close()
    return out


def run_batch(args, rank, world, local, pg):
    sec = section_batched(args, rank, world, local, pg)
    if rank == 0:
        line = {"metric": METRIC, "value": sec["value"], "unit": UNIT, "n_gpus": world, "steps": sec["steps"],
                "warmup": args.warmup, "ms_per_step": sec["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "data": "synthetic"}
        line.update({k: v for k, v in sec.items() if k not in ("value", "steps", "ms_per_step")})
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------- serving (C5)
def serve_config(args, world, kind):
    return {"workload": "serving_hex_poisson_bicgstab_ilu0", "requests": int(args.requests), "rate_per_s": args.rate,
            "m_range": [16, 128], "hbm_budget_gb": 150, "method": "BiCGStab", "preconditioner": "ILU0",
            "tol": args.tol, "server": kind, "parallelism": f"replicas{world}"}


def serve_inner(args):
    """how the GPU arm's inner solves apply ILU0 (not part of the workload's config)"""
    return {"ilu_sweeps": args.serve_sweeps, "inner_tol": args.inner_tol or "library default"}


def section_serving(args, rank, world, local, pg, nested=False):
    """Poisson-process request streams (200 req/s) of hex Poisson solves, m log-uniform in
    [16, 128], through the native server; the FP64 drop-in serves the first stream one request
    at a time.  Returns the section's dict."""
    import torch

    import elmerfem_b200 as eg
    from elmerfem_b200 import server

    torch.cuda.set_device(local)
    prm = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=args.tol, max_iter=20000,
                          inner_tol=args.inner_tol, abort_not_converged=False, ilu_sweeps=args.serve_sweeps)
    nstreams = max(1, args.serve_streams)
    streams = [server.poisson_stream(args.requests, rate=args.rate, m_lo=16, m_hi=128,
                                     seed=(1 + rank) if s == 0 else 1000 * (rank + 1) + s, sigma=1.0)
               for s in range(nstreams)]
    warm = server.poisson_stream(4, rate=1e6, m_lo=16, m_hi=24, seed=99, sigma=1.0)
    built = server.build_meshes([r.m for st in streams for r in st] + [r.m for r in warm])
    srv = server.NativeSolveServer(local, prm, hbm_budget=150e9, chunk=args.chunk)
    for mm, bm in built.items():
        srv.mesh_prototype(mm, bm)
    srv.run(warm)
    barrier(pg, None)
    stats = []
    with ClockSampler(local) as clk:
        for s, st in enumerate(streams):
            stats.append(srv.run(st, keep_solutions=(s == 0)))
    srv.close()
    reqs = streams[0]
    ctx = eg.Context(local)
    ms0 = sorted({r.m for r in reqs})
    protos = {mm: server.MeshPrototype(ctx, mm, eg.PREC_ILU0, built[mm]) for mm in ms0}
    alone = [server.Request(r.rid, r.m, r.seed, r.arrival) for r in reqs]
    fp = eg.SolverParams(method=eg.BICGSTAB, precond=eg.PREC_ILU0, tol=args.tol, max_iter=20000)
    stats64 = server.run_one_at_a_time(ctx, fp, alone, protos, keep_solutions=True)
    # converged requests only (a request that ended with an error is counted in status_counts
    # and not as a solve)
    errs = [rel(r.x, a.x) for r, a in zip(reqs, alone) if r.result.get("info") == 1]
    out = None
    if rank == 0:
        oracle = oracle_mod()
        from elmerfem_b200 import meshgen

        # against the FP64 oracle: the six smallest requests of the first stream
        pick = sorted((i for i in range(len(reqs)) if reqs[i].result.get("info") == 1),
                      key=lambda i: (reqs[i].m, i))[:6]
        eo, e64o = [], []
        for i in pick:
            r = reqs[i]
            mesh = meshgen.hex_cube(r.m)
            op = oracle.create_pattern(mesh)
            rng = np.random.Generator(np.random.PCG64(r.seed))
            k = np.exp(rng.normal(0.0, r.sigma, size=mesh.nelem))
            load = rng.random(mesh.nnodes)
            vals, rhs = oracle.assemble_poisson(mesh, op, elem_k=k, load=load)
            con = np.sort(op.perm[mesh.boundary_nodes(range(1, 7)) - 1]).astype(np.int32)
            oracle.dirichlet(op, vals, rhs, con, symmetric=False)
            xo, _ = oracle_solve_timed(op, vals, rhs, oracle.BICGSTAB, oracle.PREC_ILU0, args.tol, host_threads())
            eo.append(rel(r.x, xo))
            e64o.append(rel(alone[i].x, xo))
        cpu = None
        if world == 1 and not args.no_cpu:
            cr, cn, ct, cth = reference_systems_rate("serving", args.tol, 0, args.requests, args.rate,
                                                     args.cpu_seconds)
            cpu = {"value": cr, "unit": UNIT, "cores": cth, "kind": "port",
                   "sample": f"the first {cn} requests of the first stream, whole FP64 oracle solves one at a time "
                             f"({ct:.1f} s)"}
        for st in stats:  # solves per second count converged requests only
            st["solves_per_s"] = st["converged"] / st["makespan_s"]
        rates = [st["solves_per_s"] for st in stats]
        med = int(np.argsort(rates)[len(rates) // 2])
        s0 = stats[0]
        out = {"value": rates[med] * world, "unit": UNIT, "streams": len(stats),
               "config": serve_config(args, world, "native (egpu_server_*)"), "inner": serve_inner(args),
               "dtype": "f32 inner / f64 refinement",
               "latency_ms": {"p50": stats[med]["p50_ms"], "p99": stats[med]["p99_ms"]},
               "per_stream": stats,
               "fp64_one_at_a_time": stats64,
               "speedup_vs_fp64": s0["solves_per_s"] / stats64["solves_per_s"],
               "rel_err_vs_fp64_max": max(errs) if errs else None,
               "rel_err_vs_oracle": {"requests": pick, "m": [reqs[i].m for i in pick], "mixed_max": max(eo),
                                     "fp64_max": max(e64o), "bound": 1e-8},
               "e2e": {"value": rates[med] * world, "unit": UNIT,
                       "h2d_bytes_per_step": stats[med]["bytes_h2d"] / len(reqs),
                       "d2h_bytes_per_step": stats[med]["bytes_d2h"] / len(reqs),
                       "note": "requests submitted from host memory, solutions read back to host memory"},
               "gpu_launches": stats[med].get("kernel_launches"), "clocks": clk.summary(), "cpu_baseline": cpu}
    for P in protos.values():
        P.A.free()
    ctx.close()
    return out


def run_serve(args, rank, world, local, pg):
    sec = section_serving(args, rank, world, local, pg)
    if rank == 0:
        line = {"metric": METRIC, "value": sec["value"], "unit": UNIT, "n_gpus": world, "steps": args.requests,
                "warmup": 4, "ms_per_step": 1000.0 / (sec["value"] / world), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "data": "synthetic"}
        line.update({k: v for k, v in sec.items() if k not in ("value",)})
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson128_cg_jacobi")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--inner-tol", type=float, default=0.0, help="0: the library's choice by preconditioner")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--systems", type=int, default=512, help="batched workload: number of systems")
    ap.add_argument("--requests", type=int, default=400, help="serving workload: requests per stream")
    ap.add_argument("--serve-streams", type=int, default=3, help="serving workload: streams (median reported)")
    ap.add_argument("--serve-sweeps", type=int, default=2,
                    help="serving workload: Jacobi sweeps per ILU0 triangle in the FP32 inner solves (0: exact)")
    ap.add_argument("--batch-steps", type=int, default=3, help="nested batched section: timed batches")
    ap.add_argument("--cpu-seconds", type=float, default=6.0, help="nested sections: CPU reference sample")
    ap.add_argument("--no-nested", action="store_true", help="headline workload only")
    ap.add_argument("--rate", type=float, default=200.0, help="serving workload: mean arrivals per second")
    ap.add_argument("--chunk", type=int, default=32, help="batched/serving: inner iterations per launch")
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-tune", action="store_true", help="batched workload: skip the autotuner")
    args = ap.parse_args()
    rank, world, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, pg)
        elif args.workload == "batch512_tet_cg_jacobi":
            run_batch(args, rank, world, local, pg)
        elif args.workload == "serve_hex_bicgstab_ilu0":
            run_serve(args, rank, world, local, pg)
        else:
            run_gpu(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
