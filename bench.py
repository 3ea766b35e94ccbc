"""Benchmark of the B200 matrix-free P1 geometric-multigrid hot path.

Workload (one GPU): P1 Poisson on the unit cube split into 2x2x2 sub-cubes of 6 tetrahedra
(48 macro-cells, meshCuboid), uniformly refined to level 8 (133,432,831 inner DoFs), FP64.
One step = one V(3,3) multigrid cycle (multicolour SOR, omega = 1, linear transfers, CG on
level 0) on a seeded uniform[-1,1] right-hand side; value = finest inner DoFs per second.
Also reported: standalone kernels (apply, residual, SOR sweep, restriction, prolongation),
the roofline of the dominant kernel (cell SOR), the time to a 1e-8 relative residual of FP64
GMG against mixed precision (FP32 cycles inside FP64 defect correction) on the manufactured
problem, the variable-coefficient case to 1e-10, an end-to-end figure through host buffers,
and the reference's own CPU kernels as baseline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--level L]

With N > 1 (launched through torch.distributed.run) every rank solves an independent copy of
the problem on its GPU (the path has no inter-GPU exchange in this build: replicas only).
"""
import argparse
import concurrent.futures
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic bytes per inner DoF of the level the op writes (FP64)
BYTES = {"apply": 16, "residual": 24, "sor_sweep": 24, "restrict_per_fine": 9, "prolongate_add_per_fine": 17}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--level", type=int, default=8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--sqlite", default=None,
                   help="also append the run's figures as one row to this SQLite file (FixedSizeSQLDB rows)")
    p.add_argument("--sor-schedule", type=int, default=None, choices=[0, 1, 2, 3],
                   help="force one SOR cell-phase schedule on every level instead of autotuning (profiling runs)")
    p.add_argument("--p2-only", action="store_true",
                   help="only the P2 kernels (apply, SOR sweep, V-cycle) on P2 level LEVEL-2, one JSON line")
    p.add_argument("--sor-schedules", default=None,
                   help="FP64 schedule per level instead of autotuning, e.g. 2=3,3=1,8=0 (profiling runs, whose "
                        "serialised launches would mislead the autotuner)")
    p.add_argument("--compact", default=None,
                   help="MAX_DOFS,BLOCKS of the timed cycle's compact coarse cycle (default: the solver's own)")
    p.add_argument("--cycle-only", action="store_true",
                   help="only the kernels, autotuner and timed cycles (profiling runs); implies no serving")
    p.add_argument("--stokes-level", type=int, default=6,
                   help="P2 level of the Taylor-Hood measurements (capped at level - 2)")
    p.add_argument("--serving-requests", type=int, default=2000,
                   help="requests of the batched-serving measurement (0 skips it)")
    p.add_argument("--serving-sequential", type=int, default=400,
                   help="requests of the stream solved one at a time in FP64 (the sequential service rate)")
    return p.parse_args()


def inner_dofs(L, n=2):
    # interior lattice points of the (n 2^L + 1)^3 grid of the cube
    m = n * 2 ** L - 1
    return m ** 3


def cell_inner_dofs(L, ncells=48):
    N = 2 ** L
    return ncells * (N - 1) * (N - 2) * (N - 3) // 6


# ----------------------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = max(mx, float(c[2]))
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------------
# reference CPU kernels (oracle/_ref, compiled from the reference's own generated kernels)
# ----------------------------------------------------------------------------------------
def reference_cpu_pass(L, steps, warmup, threads):
    """Whole V(3,3) cycles of the reference's P1 multigrid on the 48-tet cube, in the reference's
    own per-primitive layout and through its generated kernels (oracle/_ref: cell and face SOR,
    face and cell apply, assign, restriction, prolongation, face <-> cell halo copies), levels L
    .. 1, on `threads` host threads. Mesh, stencils and neighbour counts come from the oracle only
    (the product library is not loaded). Returns (seconds per cycle list, inner DoFs the cycle
    updates on level L, threads used), or None without oracle/_ref."""
    from oracle import oracle
    if oracle.ref_lib() is None:
        return None
    coords, tets = oracle.cuboid_mesh((0, 0, 0), (1, 1, 1), 2, 2, 2)
    rc = oracle.RefCycle(coords, tets, L, 3, 3, seed=1)
    times, used = [], threads
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        used = rc.run(threads)
        if i >= warmup:
            times.append(time.perf_counter() - t0)
    dofs = rc.timed_dofs()
    del rc
    return times, dofs, used


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_sample_text(L):
    return ("one whole V(3,3) cycle per step on levels %d..1 of the 48-tet cube in the reference's own layout, through "
            "its generated kernels compiled from its sources (oracle/_ref): face and cell SOR, face and cell apply, "
            "r = b - Ax, restriction, prolongation, face<->cell halo copies; macro-primitives over host threads; "
            "value = cell- and face-interior DoFs of level %d (the vertex/edge phases, 0.005%% of the inner DoFs, "
            "and the level-0 CG are not run)" % (L, L))


# ----------------------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = os.environ.get("HG_BENCH_BACKEND", "nccl")  # gloo: the rank plumbing on CPU (tests)
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(v, pg):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda" if pg.get_backend() == "nccl" else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    L = args.level
    out = None
    if rank == 0:
        from oracle import oracle
        if oracle.ref_lib() is None:
            out = {"impl": "reference", "unavailable": "oracle/_ref (reference kernels) was not built"}
        else:
            thr = host_threads()
            times, dofs, thr = reference_cpu_pass(L, args.steps, args.warmup, thr)
            t = float(np.mean(times))
            v = dofs / t / 1e9
            out = {"impl": "reference", "metric": "GDoF/s", "value": v, "unit": "GDoF/s", "n_gpus": args.gpus,
                   "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
                   "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                   "config": workload_config(L),
                   "cpu_baseline": {"value": v, "unit": "GDoF/s", "cores": thr, "kind": "reference",
                                    "sample": reference_sample_text(L)},
                   "e2e": {"value": v, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def workload_config(L):
    return {"workload": "P1 Poisson GMG V(3,3) cycle, 48-tet unit cube (meshCuboid 2x2x2), level %d, FP64, "
                        "multicolour SOR omega=1, linear transfers, CG on level 0" % L,
            "level": L, "macro_cells": 48, "inner_dofs": inner_dofs(L),
            "l2": "inputs larger than L2 (%.2f GB per vector)" % (inner_dofs(L) * 8 / 1e9),
            "parallelism": "replicas"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def load_traffic(kernel, L):
    """Per-launch DRAM bytes (read + write) of `kernel` at level L, from the ncu summary
    profiles/traffic.json ({kernel: {level: bytes}}), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel, {}).get(str(L))
    except (OSError, ValueError, AttributeError):
        return None


def write_sql_row(path, out, L):
    """The run's headline figures as one row of a FixedSizeSQLDB table (the reference's result
    export, dataexport/SQL.hpp): the configuration as constant entries, the measurements as
    variable ones."""
    from hyteg_b200.sqldb import FixedSizeSQLDB
    db = FixedSizeSQLDB(path)
    db.setConstantEntry("workload", out["config"]["workload"])
    db.setConstantEntry("level", int(L))
    db.setConstantEntry("n_gpus", int(out["n_gpus"]))
    db.setConstantEntry("steps", int(out["steps"]))
    db.setVariableEntry("gdofs", float(out["value"]))
    db.setVariableEntry("ms_per_cycle", float(out["ms_per_step"]))
    db.setVariableEntry("e2e_gdofs", float(out["e2e"]["value"]))
    db.setVariableEntry("roofline_frac", float(out["roofline"]["frac"]))
    db.setVariableEntry("sm_mhz", float(out.get("clocks", {}).get("sm_mhz") or 0.0))
    db.writeRowOnRoot()


def reassembly_bench(hg, k=4, L=6, reps=5):
    """Stencil re-assembly for new macro-cell coefficients (the setup of a request in the solve
    server) on the largest serving shape, the k^3 cube of 6 k^3 macro-cells, levels 0..L: on the
    host (assembly and upload) against the device (one kernel per level from the term lists, built
    once). Wall clock around each call with the stream synchronised (both are host-issued work)."""
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), k, k, k, L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    rng = np.random.default_rng(3)
    t0 = time.perf_counter()
    A.reassemble(on_device=True)  # builds the term lists
    st.synchronize()
    t_build = time.perf_counter() - t0
    res = {}
    for name, dev in (("host", False), ("device", True)):
        ts = []
        for _ in range(reps):
            st.set_cell_coefficients(np.exp(rng.uniform(-1, 1, 6 * k ** 3)))
            st.synchronize()
            t0 = time.perf_counter()
            A.reassemble(on_device=dev)
            st.synchronize()
            ts.append(time.perf_counter() - t0)
        res[name + "_ms"] = float(np.median(ts)) * 1e3
    res.update({"mesh": "%d^3 cube, %d macro-cells, levels 0..%d" % (k, 6 * k ** 3, L),
                "term_lists_build_ms": t_build * 1e3, "speedup": res["host_ms"] / res["device_ms"]})
    return res


def serving_bench(hg, n_requests, n_sequential, seed=2024):
    """Batched serving on a seeded request stream (config 5): k in U{1..4} sub-cubes per direction
    (6..384 tets), level in U{3..6}, coefficient log-uniform in [0.1, 10], right-hand side
    uniform[-1,1] from the request's seed, tolerance 1e-8, mixed precision, Poisson arrivals. The
    first n_sequential requests are solved one after another with plain FP64 cycles (one worker):
    their service rate sets the arrival rates. One mixed-precision server (8 workers, two
    resident hierarchies per shape built ahead) then runs the whole stream at arrival rates of 2x,
    4x and 8x that sequential service rate (the last saturates it: its throughput is the server's
    capacity). Latency = completion - arrival (server clock). Setup = admission to the start of
    the solve: the stencil re-assembly for the request's coefficient on a resident hierarchy, or
    building a hierarchy when its shape has none (a request whose shape's hierarchies are all busy
    waits for one). A second server adds batched solves: every shape of levels 3-5 also gets union
    hierarchies of 2, 4 and 8 disjoint copies, in which queued requests of that shape that find no
    single hierarchy free are solved together (one launch per kernel for all of them); it runs the
    stream at 2x and 8x."""
    rng = np.random.default_rng(seed)
    reqs = [(int(rng.integers(1, 5)), int(rng.integers(3, 7)), float(np.exp(rng.uniform(np.log(0.1), np.log(10.0)))),
             int(rng.integers(1, 2 ** 62))) for _ in range(n_requests)]
    shapes = sorted({(k, L) for k, L, _, _ in reqs})

    def make(workers, precision, copies):
        srv = hg.SolveServer(workers=workers, hbm_budget_bytes=64 << 30, precision=precision)
        for _ in range(copies):
            for k, L in shapes:
                srv.prewarm(k, L)
        return srv

    def run(srv, rate, stream):
        arr = np.cumsum(rng.exponential(1.0 / rate, len(stream))) if rate else np.zeros(len(stream))
        t0 = time.perf_counter()
        ids = []
        for (k, L, c, sd), ta in zip(stream, arr):
            d = ta - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(k, L, c, sd, 1e-8, 100))
        for i in ids:
            srv.wait(i)
        res = [srv.result(i) for i in ids]
        st = srv.stats()
        lat = np.array([r["t_end"] - r["t_submit"] for r in res])
        span = max(r["t_end"] for r in res) - min(r["t_submit"] for r in res)
        dofs = sum(r["inner_dofs"] for r in res)
        setup = np.array([r["t_solve"] - r["t_start"] for r in res])
        built = np.array([r["built_hierarchy"] for r in res])
        bsz = np.array([r["batch_size"] for r in res])
        return {"requests": len(res), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "seconds": span, "gdofs": dofs / span / 1e9,
                "max_rel_residual": max(r["rel_residual"] for r in res),
                "mean_iterations": float(np.mean([r["iterations"] for r in res])), "peak_bytes": st["peak_bytes"],
                "mean_setup_ms": float(setup.mean() * 1e3),
                "hierarchies_built_on_admission": int(built.sum()),
                "mean_setup_ms_resident": float(setup[~built].mean() * 1e3) if (~built).any() else None,
                "mean_setup_ms_built": float(setup[built].mean() * 1e3) if built.any() else None,
                "mean_solve_ms": float(np.mean([r["t_end"] - r["t_solve"] for r in res]) * 1e3),
                "requests_batched": int((bsz > 1).sum()), "mean_batch_size": float(bsz.mean())}

    srv = make(1, 8, 1)
    seq = run(srv, 0, reqs[:n_sequential])  # all submitted at once, one worker: sequential FP64 solves
    srv.close()
    mu = seq["requests"] / seq["seconds"]
    out = {"workload": "%d seeded requests: k in U{1..4}, level in U{3..6}, coefficient log-U[0.1,10], "
                       "tol 1e-8, Poisson arrivals; the sequential FP64 rate from its first %d"
                       % (n_requests, n_sequential),
           "sequential_fp64": seq}
    srv = make(8, 4, 2)  # resident hierarchies: two per shape, kept across the three runs
    for mult in (2.0, 4.0, 8.0):
        out["mixed_rate_%gx" % mult] = dict(run(srv, mult * mu, reqs), arrival_rate_per_s=mult * mu)
    srv.close()
    out["capacity_vs_sequential"] = out["mixed_rate_8x"]["gdofs"] / seq["gdofs"]
    # batched solves: the shapes of levels 3-5 also get union hierarchies of 2, 4 and 8 copies;
    # two or more queued requests of such a shape that find no single hierarchy free are solved
    # together in the smallest idle union that takes them all
    t0 = time.perf_counter()
    srv = make(8, 4, 2)
    for k, L in shapes:
        if L <= 5:
            for copies in (2, 4, 8):
                srv.prewarm_batch(k, L, copies)
    srv.set_batching(5)
    out["batched_prewarm_seconds"] = time.perf_counter() - t0
    for mult in (2.0, 8.0):
        out["batched_rate_%gx" % mult] = dict(run(srv, mult * mu, reqs), arrival_rate_per_s=mult * mu)
    srv.close()
    out["batched_capacity_vs_sequential"] = out["batched_rate_8x"]["gdofs"] / seq["gdofs"]
    return out


def p2_kernels(hg, st, L2, timed):
    """P2 Laplace on P2 level L2 of the same cube (its DoFs are the vertex lattice L2 + 1):
    apply, multicolour SOR sweep, one P2 V(3,3) cycle; FP64. Algorithmic bytes of the apply:
    16 per inner P2 DoF (read x, write y)."""
    Inner = hg.Inner | hg.NeumannBoundary
    n_in = inner_dofs(L2 + 1)
    A = hg.P2ConstantLaplaceOperator(st, 0, L2)
    x, b, y = (hg.P2Function(nm, st, 0, L2) for nm in ("p2x", "p2b", "p2y"))
    x.fill_random(5, L2, hg.Inner)
    b.fill_random(6, L2, hg.Inner)
    t_apply = timed(lambda: A.apply(x, y, L2, hg.Inner), 5)
    t_sor = timed(lambda: A.smooth_sor(x, b, 1.0, L2, Inner), 3)
    g = hg.P2GeometricMultigridSolver(st, A, 0, L2, 3, 3, 1.0)
    t_cycle = timed(lambda: g.solve(x, b, L2), 2, warm=4)  # past the solver's graph capture
    import torch
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("p2_ops")  # one sweep and one apply, for a launch list
    A.smooth_sor(x, b, 1.0, L2, Inner)
    A.apply(x, y, L2, hg.Inner)
    st.synchronize()
    torch.cuda.nvtx.range_pop()
    return {"p2_level": L2, "inner_dofs": n_in,
            "apply": {"ms": t_apply * 1e3, "gdofs": n_in / t_apply / 1e9, "GBs_algorithmic": 16 * n_in / t_apply / 1e9},
            "sor_sweep": {"ms": t_sor * 1e3, "gdofs": n_in / t_sor / 1e9},
            "vcycle": {"ms": t_cycle * 1e3, "gdofs": n_in / t_cycle / 1e9}}


def stokes_bench(hg, st, L2):
    """P2-P1 Taylor-Hood lid-driven cavity on P2 level L2 of the same cube (velocity on the
    vertex lattice L2 + 1, pressure on L2): MINRES to 1e-8 with the block-diagonal multigrid
    preconditioner (symmetric P2 V(2,2) per velocity component, lumped P1 mass), the V-cycles in
    FP64 and in FP32 (mixed); residual and update in FP64. Then ten V(3,3) cycles of the multigrid
    on the whole system with the Uzawa smoother (three velocity sweeps), its relaxation estimated
    by power iteration."""
    import torch
    xyz, _ = st.host().slot_info(L2 + 1)
    lid = np.where(np.abs(xyz[:, 2] - 1.0) < 1e-12, 1.0, 0.0)
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, L2)
    out = {"p2_level": L2, "velocity_dofs": 3 * inner_dofs(L2 + 1), "pressure_dofs": (2 * 2 ** L2 + 1) ** 3,
           "problem": "lid-driven cavity, u = (1,0,0) on z = 1, no slip elsewhere, zero-mean pressure"}
    sol = {}
    for name, dt in (("fp64", np.float64), ("mixed", np.float32)):
        u = [hg.P2Function("su%d" % k, st, 0, L2) for k in range(3)]
        f = [hg.P2Function("sf%d" % k, st, 0, L2) for k in range(3)]
        p, g = hg.P1Function("sp", st, 0, L2), hg.P1Function("sg", st, 0, L2)
        u[0].from_numpy(L2, lid)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, rel, _ = S.minres(u, p, f, g, L2, nu=2, max_iter=500, tol=1e-8, precondition_dtype=dt)
        torch.cuda.synchronize()
        out[name] = {"iterations": it, "seconds": time.perf_counter() - t0, "rel_residual": rel}
        sol[name] = [x.to_numpy(L2) for x in u]
    out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    out["max_velocity_difference_mixed_vs_fp64"] = float(max(np.abs(a - b).max() for a, b in zip(sol["fp64"],
                                                                                                   sol["mixed"])))
    # multigrid on the whole system with the Uzawa smoother (relaxation from 20 power iterations)
    t0 = time.perf_counter()
    omega = hg.estimateUzawaRelaxationParameter(st, S, L2, 20, 3)
    torch.cuda.synchronize()
    t_est = time.perf_counter() - t0
    sm = hg.UzawaSmoother(st, S, 0, L2, omega, 3)
    mg = hg.StokesGeometricMultigridSolver(st, S, sm, 0, L2, 3, 3)
    u = [hg.P2Function("zu%d" % k, st, 0, L2) for k in range(3)]
    f = [hg.P2Function("zf%d" % k, st, 0, L2) for k in range(3)]
    p, g = hg.P1Function("zp", st, 0, L2), hg.P1Function("zg", st, 0, L2)
    u[0].from_numpy(L2, lid)
    mg.solve(u, p, f, g, L2)  # builds the coarse pseudo-inverse
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    it, rel, hist = mg.solve_to(u, p, f, g, L2, 1e-30, 10)
    torch.cuda.synchronize()
    t_cyc = (time.perf_counter() - t0) / max(it, 1)
    out["uzawa_multigrid"] = {"omega_estimate": omega, "estimate_seconds": t_est, "cycle": "V(3,3), 3 velocity sweeps",
                              "ms_per_cycle": t_cyc * 1e3, "cycles": it,
                              "convergence_factors": [float(a / b) for a, b in zip(hist[1:], hist[:-1])]}
    return out


def fp32_kernels(hg, st, A, x, b, L, Inner, N_in, Nc, timed):
    """The same kernels on FP32 copies of the vectors (the arithmetic of the inner cycles of the
    mixed-precision solve), and one FP32 V(3,3) cycle. Algorithmic bytes are half the FP64 ones."""
    xf = hg.P1Function("xf", st, 0, L, dtype=np.float32)
    bf = hg.P1Function("bf", st, 0, L, dtype=np.float32)
    rf = hg.P1Function("rf", st, L, L, dtype=np.float32)
    xf.copy_from(x, L)
    bf.copy_from(b, L)
    t = {"apply": timed(lambda: A.apply(xf, rf, L, Inner), 5),
         "residual": timed(lambda: A.residual(xf, bf, rf, L, Inner), 5),
         "sor_sweep": timed(lambda: A.smooth_sor(xf, bf, 1.0, L, Inner), 4)}
    t_cells = timed(lambda: A.smooth_sor_primitives(xf, bf, 1.0, L, Inner, kinds=1 << hg.CELL, refresh=False), 4)
    g = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                    hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3,
                                    dtype=np.float32)
    # a new solver's first cycles run eagerly (they allocate its buffers) and the next one is
    # captured into a graph: warm up past the capture so that only replays are timed
    t_cycle = timed(lambda: g.solve(A, xf, bf, L), 3, warm=4)
    out = {k: {"ms": v * 1e3, "GBs_algorithmic": BYTES[k] / 2 * N_in / v / 1e9} for k, v in t.items()}
    out["cell_sor_single_pass"] = {"ms": t_cells * 1e3, "GBs_algorithmic": BYTES["sor_sweep"] / 2 * Nc / t_cells / 1e9}
    out["vcycle"] = {"ms": t_cycle * 1e3}
    return out


def time_to_solution(hg, st, A, L, N_in, Inner):
    """Manufactured problem -Lap u = 3 pi^2 u, u = sin(pi x) sin(pi y) sin(pi z), b = M I(f), x0 = 0:
    FP64 V(3,3) cycles vs FP64 defect correction around FP32 V(3,3) cycles, each to a 1e-8
    relative residual; then the variable-coefficient case k(x) = 1 + 0.5 sin(2 pi x) cos(2 pi y) z
    (piecewise constant per macro-cell) to 1e-10. Errors are discrete L2 (RMS over inner DoFs)."""
    import torch
    M = hg.P1ConstantMassOperator(st, L, L)
    f = hg.P1Function("f", st, L, L)
    u = hg.P1Function("u", st, L, L)
    e = hg.P1Function("e", st, L, L)
    bm = hg.P1Function("bm", st, 0, L)
    xs = hg.P1Function("xs", st, 0, L)
    x64 = hg.P1Function("x64", st, L, L)
    u.interpolate_sines(1.0, 1.0, L)
    f.interpolate_sines(3 * np.pi ** 2, 1.0, L)
    M.apply(f, bm, L, Inner)
    del M, f

    def rms(a, b_=None):
        if b_ is not None:
            e.assign([1.0, -1.0], [a, b_], L, Inner)
            a = e
        return float(np.sqrt(a.dotGlobal(a, L, Inner) / N_in))

    def run(op, rhs, dtype, tol):
        g = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                        hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3,
                                        dtype=dtype)
        xs.interpolate(0.0, L, hg.All)
        g.solve_to(op, xs, rhs, L, tol, 2)       # warm-up: workspace allocation, first launches
        xs.interpolate(0.0, L, hg.All)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, rel, hist = g.solve_to(op, xs, rhs, L, tol, 100)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        del g
        factors = [float(hist[0])] + [float(hist[i + 1] / hist[i]) for i in range(len(hist) - 1)]
        return {"iterations": it, "seconds": dt, "final_rel_residual": rel, "convergence_factors": factors}

    out = {"problem": "manufactured u = sin(pi x) sin(pi y) sin(pi z), b = M I(3 pi^2 u), x0 = 0, Dirichlet 0",
           "target_rel_residual": 1e-8, "error_norm": "discrete L2 (RMS over inner DoFs)"}
    r64 = run(A, bm, np.float64, 1e-8)
    r64["err_vs_manufactured"] = rms(xs, u)
    x64.assign([1.0], [xs], L, hg.All)
    r32 = run(A, bm, np.float32, 1e-8)
    r32["err_vs_manufactured"] = rms(xs, u)
    r32["err_vs_fp64_solve"] = rms(xs, x64) / rms(x64)
    out["fp64"], out["mixed"] = r64, r32
    out["speedup_mixed_vs_fp64"] = r64["seconds"] / r32["seconds"]

    # variable coefficient, 1e-10 (errors against the FP64 GPU solve)
    mesh = st.host()
    nc = mesh.counts()[3]
    cent = np.array([np.mean([mesh.primitive(hg.VERTEX, v)[1] for v in mesh.primitive(hg.CELL, c)[0]], axis=0)
                     for c in range(nc)])
    st.set_cell_coefficients(1.0 + 0.5 * np.sin(2 * np.pi * cent[:, 0]) * np.cos(2 * np.pi * cent[:, 1]) * cent[:, 2])
    Ak = hg.P1ConstantLaplaceOperator(st, 0, L)
    # With k piecewise constant, the smooth u above does not satisfy the flux conditions across
    # the macro-cell interfaces, so it is no solution of -div(k grad u) = f. The manufactured
    # solution is therefore discrete: b = A_k I(u), whose exact discrete solution is I(u).
    bm.interpolate(0.0, L, hg.All)
    Ak.apply(u, bm, L, Inner)
    v64 = run(Ak, bm, np.float64, 1e-10)
    v64["err_vs_manufactured"] = rms(xs, u) / rms(u)
    x64.assign([1.0], [xs], L, hg.All)
    v32 = run(Ak, bm, np.float32, 1e-10)
    v32["err_vs_manufactured"] = rms(xs, u) / rms(u)
    v32["err_vs_fp64_solve"] = rms(xs, x64) / rms(x64)
    out["variable_k"] = {"k": "1 + 0.5 sin(2 pi x) cos(2 pi y) z at macro-cell centroids", "target_rel_residual": 1e-10,
                         "problem": "b = A_k I(u), u = sin(pi x) sin(pi y) sin(pi z): the manufactured discrete solution "
                                    "is I(u); errors are relative discrete L2 (RMS over inner DoFs)",
                         "fp64": v64, "mixed": v32, "speedup_mixed_vs_fp64": v64["seconds"] / v32["seconds"]}
    del Ak
    st.set_cell_coefficients(np.ones(nc))
    return out


def convergence_by_level(hg, st, L, cycles=20):
    """Per-level V(3,3) convergence on the manufactured problem (b = M I(3 pi^2 u), x0 = 0, CG on
    level 0): the residual factor of each of `cycles` cycles on levels 3 .. L, the mean of the
    first ten and the asymptotic factor (geometric mean of cycles 15-20, or of the last six above
    the rounding floor of the residual)."""
    inn = hg.Inner | hg.NeumannBoundary
    out = {}
    for lv in range(3, L + 1):
        A = hg.P1ConstantLaplaceOperator(st, 0, lv)
        M = hg.P1ConstantMassOperator(st, lv, lv)
        x, b, r, f = (hg.P1Function(n, st, 0, lv) for n in ("cx", "cb", "cr", "cf"))
        f.interpolate_sines(3 * np.pi ** 2, 1.0, lv)
        M.apply(f, b, lv, hg.Inner)
        g = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                        hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, lv, 3, 3)

        def res():
            A.residual(x, b, r, lv, inn)
            return float(np.sqrt(r.dotGlobal(r, lv, inn)))

        h = [res()]
        for _ in range(cycles):
            g.solve(A, x, b, lv)
            h.append(res())
        fac = [h[i + 1] / h[i] for i in range(cycles)]
        above = [i for i in range(cycles) if h[i + 1] / h[0] > 1e-12]
        tail = above[-6:] if len(above) >= 6 else list(range(cycles - 6, cycles))
        out[str(lv)] = {"factors": fac, "mean_first_10": float(np.exp(np.mean(np.log(fac[:10])))),
                        "asymptotic": float(np.exp(np.mean(np.log([fac[i] for i in tail])))),
                        "asymptotic_cycles": [tail[0] + 1, tail[-1] + 1]}
        del g, A, M, x, b, r, f
    return out


def run_ours(args):
    import torch
    import hyteg_b200 as hg

    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    L = args.level
    N_in = inner_dofs(L)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    st.set_stream(stream.cuda_stream)

    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x = hg.P1Function("x", st, 0, L)
    b = hg.P1Function("b", st, 0, L)
    r = hg.P1Function("r", st, 0, L)
    t = hg.P1Function("t", st, 0, L)
    n = st.level_size(L)
    rng = np.random.default_rng(42 + rank)
    host_b = torch.empty(n, dtype=torch.float64, pin_memory=True)
    host_b.numpy()[:] = rng.uniform(-1.0, 1.0, n)
    b.from_numpy(L, host_b.numpy())
    b.communicate(L)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    if args.compact:
        gmg.set_compact(A, *(int(v) for v in args.compact.split(",")))
    Inner = hg.Inner | hg.NeumannBoundary

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed(fn, reps, warm=2):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e-3

    if args.p2_only:  # profiling runs of the P2 path alone
        if rank == 0:
            print(json.dumps({"p2": p2_kernels(hg, st, L - 2, timed)}), flush=True)
        return

    # --- standalone kernels on the seeded source vector ----------------------------------
    x.from_numpy(L, host_b.numpy())
    kern = {}
    kern["apply"] = timed(lambda: A.apply(x, r, L, Inner), 5)
    kern["residual"] = timed(lambda: A.residual(x, b, r, L, Inner), 5)
    kern["sor_sweep"] = timed(lambda: A.smooth_sor(x, b, 1.0, L, Inner), 3)
    kern["restrict"] = timed(lambda: hg.P1toP1LinearRestriction().restrict(r, L, Inner), 5)
    kern["prolongate_add"] = timed(lambda: hg.P1toP1LinearProlongation().prolongateAndAdd(x, L - 1, Inner), 5)
    kern["halo_refresh"] = timed(lambda: x.communicate(L), 5)
    # dominant kernel alone: the cell phase of the SOR sweep (one single-pass launch plus the copy
    # of the face/edge/vertex arrays into the exchanged buffer), and cell apply
    t_sor_cells = timed(lambda: A.smooth_sor_primitives(x, b, 1.0, L, Inner, kinds=1 << hg.CELL, refresh=False), 4)
    t_apply_cells = timed(lambda: A.apply_primitives(x, r, L, Inner, kinds=1 << hg.CELL, refresh=False), 5)
    st.set_sor_schedule(1)    # the four in-place colour passes, for comparison
    t_sor_passes = timed(lambda: A.smooth_sor_primitives(x, b, 1.0, L, Inner, kinds=1 << hg.CELL, refresh=False), 2)
    kern["sor_sweep_colour_passes"] = timed(lambda: A.smooth_sor(x, b, 1.0, L, Inner), 2)
    st.set_sor_schedule(0)
    Nc = cell_inner_dofs(L)
    kernels = {k: {"ms": v * 1e3, "gdofs": N_in / v / 1e9} for k, v in kern.items()}
    for k in ("apply", "residual", "sor_sweep", "sor_sweep_colour_passes"):
        kernels[k]["GBs_algorithmic"] = BYTES[k.replace("_colour_passes", "")] * N_in / kern[k] / 1e9
    kernels["cell_sor_single_pass"] = {"ms": t_sor_cells * 1e3,
                                       "GBs_algorithmic": BYTES["sor_sweep"] * Nc / t_sor_cells / 1e9}
    kernels["cell_sor_colour_passes"] = {"ms": t_sor_passes * 1e3,
                                         "GBs_algorithmic": BYTES["sor_sweep"] * Nc / t_sor_passes / 1e9}
    kernels["cell_apply_launch"] = {"ms": t_apply_cells * 1e3, "GBs_algorithmic": BYTES["apply"] * Nc / t_apply_cells / 1e9}
    if not args.cycle_only:
        kernels["fp32"] = fp32_kernels(hg, st, A, x, b, L, Inner, N_in, Nc, timed)
    if L >= 3 and not args.cycle_only:
        kernels["p2"] = p2_kernels(hg, st, L - 2, timed)
        kernels["stokes"] = stokes_bench(hg, st, min(L - 2, args.stokes_level))
        if min(L - 2, args.stokes_level) > 5:  # the smaller Stokes case (P2 level 5) beside it
            kernels["stokes_p2_level_5"] = stokes_bench(hg, st, 5)
    if not args.cycle_only:
        kernels["reassembly"] = reassembly_bench(hg)

    # --- autotuner: the faster SOR schedule per level and precision, used from here on
    autotune = {}
    if args.sor_schedule is not None:
        st.set_sor_schedule(args.sor_schedule)
        autotune = {"forced_schedule": args.sor_schedule}
    if args.sor_schedules:
        picks = {int(a): int(b) for a, b in (kv.split("=") for kv in args.sor_schedules.split(","))}
        for lv, sch in picks.items():
            st.set_sor_schedule_level(lv, sch, np.float64)
        autotune = {"forced_schedules_fp64": {str(k): v for k, v in picks.items()}}
    for name, dt in (("fp64", np.float64), ("fp32", np.float32)):
        if args.sor_schedule is not None or args.sor_schedules:
            break
        picks = st.autotune_sor(2, L, dtype=dt, reps=3)
        autotune[name] = {str(lv): {"schedule": c, "ms_single_pass": t0, "ms_colour_passes": t1,
                                    "ms_single_pass_short_tiles": t2, "ms_colour_split": t3}
                          for lv, (c, t0, t1, t2, t3) in picks.items()}

    # --- time to solution: FP64 GMG vs mixed precision (FP32 cycles inside FP64 defect correction)
    solve = None if args.cycle_only else time_to_solution(hg, st, A, L, N_in, Inner)
    if solve is not None:
        solve["convergence_by_level"] = convergence_by_level(hg, st, L)
    x.from_numpy(L, host_b.numpy())

    # --- the timed region: K V(3,3) cycles --------------------------------------------------
    for _ in range(args.warmup):
        gmg.solve(A, x, b, L)
    launches0 = st.launch_count()
    barrier(pg)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0, e1 = ev(), ev()
        torch.cuda.nvtx.range_push("timed_cycles")   # launch-list filter for ncu --nvtx-include
        e0.record(stream)
        for _ in range(args.steps):
            gmg.solve(A, x, b, L)
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    t_steps = e0.elapsed_time(e1) * 1e-3
    launches = st.launch_count() - launches0
    barrier(pg)
    t_max = max_over_ranks(t_steps, pg)
    ms = t_max / args.steps * 1e3
    value = world * N_in * args.steps / t_max / 1e9

    # --- end to end through the public API with host buffers --------------------------------
    # Every step uploads its right-hand side from pinned host memory, runs one V(3,3) cycle, and
    # downloads the step's result -- the solution x -- into pinned host memory, both as the packed
    # owned DoFs of the level (every DoF once; hg_function_*_owned_async). Two (x, b) pairs
    # alternate. Per step, in this order: the cycle on its pair; the download of its solution
    # (packed on the storage's stream behind the cycle, copied on one copy stream); the upload of
    # the next step's right-hand side into the other pair (copied on a second copy stream while the
    # cycle runs, unpacked behind it). The library orders each staging buffer's uses by events.
    # The first upload and the last download are not overlapped.
    x2 = hg.P1Function("x2", st, 0, L)
    b2 = hg.P1Function("b2", st, 0, L)
    xs2, bs2 = (x, x2), (b, b2)
    slots = st.host().owned_slots(L)
    n_own = len(slots)
    assert st.owned_count(L) == n_own
    host_bo = torch.empty(n_own, dtype=torch.float64, pin_memory=True)
    host_bo.numpy()[:] = host_b.numpy()[slots]
    host_x = [torch.empty(n_own, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    for bb in (b, b2):  # both right-hand sides set, then the second pair's cycles run eagerly and get a graph
        bb.upload_owned_async(L, host_bo.numpy(), up.cuda_stream)
    torch.cuda.synchronize()
    for _ in range(3):
        gmg.solve(A, x2, b2, L)
        xs2[1].download_owned_async(L, host_x[1].numpy(), down.cuda_stream)
    torch.cuda.synchronize()
    barrier(pg)
    e0, e1 = ev(), ev()
    e0.record(stream)
    up.wait_stream(stream)
    down.wait_stream(stream)
    bs2[0].upload_owned_async(L, host_bo.numpy(), up.cuda_stream)
    for k in range(args.steps):
        cur = k % 2
        gmg.solve(A, xs2[cur], bs2[cur], L)
        xs2[cur].download_owned_async(L, host_x[cur].numpy(), down.cuda_stream)
        if k + 1 < args.steps:
            bs2[1 - cur].upload_owned_async(L, host_bo.numpy(), up.cuda_stream)
    stream.wait_stream(down)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) * 1e-3, pg)
    e2e_finite = bool(np.isfinite(host_x[(args.steps - 1) % 2].numpy()[:1000]).all())
    # the host link alone, outside the timed region: one step's download and upload issued
    # together on the two copy streams, in the loop's order (the pipelined loop overlaps exactly
    # these with a cycle)
    def copies():
        xs2[0].download_owned_async(L, host_x[0].numpy(), down.cuda_stream)
        bs2[1].upload_owned_async(L, host_bo.numpy(), up.cuda_stream)
    copies()
    torch.cuda.synchronize()
    c0, c1 = ev(), ev()
    c0.record(stream)
    for _ in range(3):
        up.wait_stream(stream)
        down.wait_stream(stream)
        copies()
        stream.wait_stream(up)
        stream.wait_stream(down)
    c1.record(stream)
    torch.cuda.synchronize()
    t_link = c0.elapsed_time(c1) * 1e-3 / 3
    del x2, b2

    # --- where one cycle's time goes: the solver's timing tree (device events, eager cycle) ----
    gmg.set_timing(A, True)
    gmg.solve(A, x, b, L)
    tree = gmg.timing_tree(A)["Geometric Multigrid Solver"]
    gmg.set_timing(A, False)
    cycle_tree = {"total_ms": tree["total"] * 1e3, "levels": {}}
    for lv in range(L + 1):
        node = tree.get("Level %d" % lv, {})
        cycle_tree["levels"][str(lv)] = {k: node[k]["total"] * 1e3 for k in
                                         ("Smoother", "Restriction", "Prolongation", "Coarse Grid Solver",
                                          "Remainder") if k in node}

    peak, peak_kind = load_peaks()
    achieved = BYTES["sor_sweep"] * Nc / t_sor_cells / 1e9
    traffic = load_traffic("cellSorWaveKernel<double, 0>", L)
    out = {
        "metric": "GDoF/s", "value": value, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform[-1,1] right-hand side)",
        "config": workload_config(L),
        "roofline": {"kernel": "cellSorWaveKernel<double, 0> (cell-interior multicolour SOR sweep, one launch; timed "
                               "with the copy of the non-cell arrays into the exchanged buffer)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": BYTES["sor_sweep"] * Nc},
        "e2e": {"value": world * N_in * args.steps / t_e2e / 1e9, "unit": "GDoF/s", "h2d_bytes_per_step": n_own * 8,
                "d2h_bytes_per_step": n_own * 8, "ms_per_step": t_e2e / args.steps * 1e3,
                "result_downloaded": "the solution x every step: all %d DoFs of level %d, packed (finite: %s)"
                                     % (n_own, L, e2e_finite),
                "pipelining": "two (x, b) pairs alternate: per step the cycle, the download of its solution "
                              "(packed behind the cycle, one copy stream) and the upload of the next right-hand "
                              "side (second copy stream, overlapping the cycle; unpacked behind it); the first "
                              "upload and the last download are not overlapped",
                "host_link_ms_per_step": t_link * 1e3,
                "host_link_GBs_per_direction": n_own * 8 / t_link / 1e9,
                "bound_ms_per_step": (max(t_link, t_max / args.steps) * (args.steps - 1) + 2 * t_link
                                      + t_max / args.steps) / args.steps * 1e3,
                "bound_note": "one step's upload and download together (host_link_ms_per_step) against the "
                              "device cycle: steps - 1 pipelined periods of the slower of the two, plus the "
                              "unoverlapped first upload, last cycle and last download, per step"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "kernels": kernels,
        "solve": solve,
        "autotune_sor": autotune,
        # levels 0 .. compact_top of every timed cycle run as one launch (the compact coarse
        # cycle); the timing tree below times the level-by-level cycle
        "compact_top": gmg.compact_top(A),
        "timing_tree_one_cycle_ms": cycle_tree,
    }
    if world == 1 and args.serving_requests > 0 and not args.cycle_only:
        out["serving"] = serving_bench(hg, args.serving_requests, min(args.serving_sequential, args.serving_requests))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        thr = host_threads()
        ref = reference_cpu_pass(L, 5, 1, thr)  # median of five cycles on all host threads
        if ref:
            times, dofs, thr = ref
            out["cpu_baseline"] = {"value": dofs / statistics.median(times) / 1e9, "unit": "GDoF/s",
                                   "cores": thr, "kind": "reference", "repeats": len(times),
                                   "sample": reference_sample_text(L)}
            one = reference_cpu_pass(L, 1, 0, 1)  # and one cycle on a single core
            if one:
                out["cpu_baseline"]["single_core_value"] = one[1] / one[0][0] / 1e9
    if rank == 0:
        print(json.dumps(out), flush=True)
        if args.sqlite:
            write_sql_row(args.sqlite, out, L)
    del gmg
    if pg is not None:
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
