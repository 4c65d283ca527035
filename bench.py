"""Benchmark: 2048^2 variable-coefficient Poisson solve to max residual 1e-6.

Workload (seeded synthetic input, the reference publishes no data set): the
two-phase projection problem on a 2048x2048 uniform grid (depth 11) --
face alpha = 1/rho with rho = 1 inside a circle of radius 0.25 and 1000
outside, blended by tanh over 2 cells; b ~ N(0, 1) per cell; Dirichlet a = 0
on the four walls (basilisk_b200.problems.two_phase_2d).  One step = one
poisson() solve from a = 0 to max|residual| <= 1e-6, as the reference's
mg_solve does it (V-cycles, nrelax adaptation).

Headline: the mixed form (FP32 cycles, FP64 iterative refinement), in
solves/s; the plain FP64 form is measured beside it on the same input.
Inputs live in HBM and exceed L2 (a, b, alpha_x, alpha_y and the hierarchy:
~400 MB), and L2 is also flushed (a 256 MB write) before every timed step,
outside the step's event pair.

Under torchrun (N > 1) every rank solves its own instance (replicas: the
solve does not shard); value = N * solves / max-over-ranks
time.

--impl reference times the reference algorithm's CPU implementation (the
plain-C restatement in oracle/, OpenMP on all host threads, lexicographic
Gauss-Seidel as the reference's default relax): full solves of the same
workload (about 20 s each on 8 cores).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("time-to-residual 1e-6 & V-cycle HBM GB/s, 2048²: mixed vs FP64 mg_solve, 1 B200")
DEPTH = 11
TOL = 1e-6


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# dram__bytes_read.sum + dram__bytes_write.sum of one k_relax_tile2d_w launch on
# the 2048^2 level (ncu, 102.2 + 18.2 MB, the first launch of a cycle's finest
# level, cold)
TILE_LAUNCH_DRAM_BYTES = 120.4e6


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def window(self, t0, t1):
        """Keep only the samples read between t0 and t1 (time.monotonic()):
        the sampler is started before the warm-up, so that nvidia-smi's own
        start-up does not fall inside the timed region."""
        self.t0, self.t1 = t0, t1

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device_index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [l for t, l in self.lines
                 if self.t0 is None or self.t0 <= t <= self.t1 + 0.25]
        if not lines:
            lines = [l for _, l in self.lines[-1:]]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        busy = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(backend=None, timeout_s=600):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): NCCL
    with a device, gloo without one (the host-side tests).  The replicas
    exchange nothing but the barrier and the maximum of their times."""
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    """The maximum of v over the ranks (the slowest replica's time)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Solver:
    """The workload on one grid: fields created once, reset every step."""

    def __init__(self, prob, precision, relax="rbgs"):
        import torch
        import basilisk_b200 as bmg
        from basilisk_b200 import problems
        self.torch = torch
        self.g = bmg.Grid(2, prob["depth"], relax=relax, precision=precision)
        self.g.set_stream(torch.cuda.current_stream().cuda_stream)
        self.a, self.b, self.alpha, self.lam = problems.setup(self.g, prob)
        n = 1 << prob["depth"]
        self.zero = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        self.g.set_timing(True)

    def step(self):
        self.a.set(self.zero)
        return self.g.poisson(self.a, self.b, alpha=self.alpha, lambda_=self.lam, tolerance=TOL)


def flush_l2(buf):
    buf.zero_()


def time_steps(solver, steps, warmup, ws, flush, clocks=None):
    import torch
    for _ in range(warmup):
        solver.step()
    torch.cuda.synchronize()
    barrier(ws)
    solver.g.reset_counters()
    times, stats = [], None
    t_begin = time.monotonic()
    for _ in range(steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        stats = solver.step()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    if clocks is not None:
        clocks.window(t_begin, time.monotonic())
    barrier(ws)
    return times, stats, solver.g.counters()


def e2e_steps(prob, steps, warmup, precision):
    """The public API with host buffers: every step copies the inputs
    (a = 0, b, alpha_x, alpha_y) from pinned host memory to the device, solves,
    and reads the solution back to pinned host memory."""
    import torch
    import basilisk_b200 as bmg
    g = bmg.Grid(2, prob["depth"], relax="rbgs", precision=precision)
    g.set_stream(torch.cuda.current_stream().cuda_stream)
    a = g.scalar()
    for side, (kind, val) in prob["bc"].items():
        a.bc(side, kind, val)
    b = g.scalar()
    alpha = g.face_vector()
    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
    h_b = pin(prob["b"])
    h_ax, h_ay = pin(prob["alpha"][0]), pin(prob["alpha"][1])
    h_a0 = pin(np.zeros_like(prob["b"]))
    h_out = torch.empty_like(h_b).pin_memory()
    L = bmg._lib.load()

    def put(f, h):
        bmg._lib.check(L.bmg_field_set(g.ptr, f.scalar, h.data_ptr(), h.numel(), bmg._lib.HOST))

    def one():
        put(a, h_a0); put(b, h_b)
        put(alpha.components[0], h_ax); put(alpha.components[1], h_ay)
        st = g.poisson(a, b, alpha=alpha, tolerance=TOL)
        bmg._lib.check(L.bmg_field_get(g.ptr, a.scalar, h_out.data_ptr(), h_out.numel(),
                                       bmg._lib.HOST))
        return st

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        one()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    h2d = sum(x.numel() * 8 for x in (h_a0, h_b, h_ax, h_ay))
    d2h = h_out.numel() * 8
    g.close()
    return times, h2d, d2h


def cpu_solve(prob, threads=None):
    """One full solve of the workload by the oracle (plain-C restatement of
    the reference's mg_solve, OpenMP on all host threads, the reference's
    default lexicographic Gauss-Seidel relax).  Returns (seconds, mgstats)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import oracle
    from helpers import oracle_grid
    threads = threads or os.cpu_count()
    g = oracle_grid(prob, relax=oracle.RELAX_GS, threads=threads)
    t0 = time.perf_counter()
    st = g.poisson(tolerance=TOL)
    return time.perf_counter() - t0, st, threads


def oracle_floor(prob, threads=None):
    """The oracle's red-black solve of the workload driven to its residual
    floor: to 1e-9, then on to 3e-10 (further cycles stall above 2e-10 while
    nrelax climbs to 100).  Returns (solution at the floor, its max residual,
    the 1e-9 iterate)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import oracle
    from helpers import oracle_grid
    threads = threads or os.cpu_count()
    oracle.set_globals(2, nitermax=400)
    try:
        g = oracle_grid(prob, relax=oracle.RELAX_RBGS, threads=threads)
        g.poisson(tolerance=1e-9)
        a9 = g.get_a()
        st = g.poisson(tolerance=3e-10)
        return g.get_a(), st["resa"], a9
    finally:
        oracle.set_globals(2, nitermax=100)


def run_workload(args, ws, rank, local):
    """The other workloads of the scope table, one JSON line each (not the
    headline): the quadtree problem (two_phase_tree, depth 11), the 3D
    periodic Helmholtz problem (helmholtz_3d, 256^3), one step = one
    poisson () solve from a = 0; and the differentiable batch
    (random_field_batch, 16 x 512^2), one step = a forward and backward pass
    through basilisk_b200.autograd."""
    import torch
    import basilisk_b200 as bmg
    from basilisk_b200 import problems
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    clocks = ClockSampler(local)
    if args.workload == "two_phase_tree":
        g = bmg.TreeGrid(11, relax="rbgs", precision=args.precision)
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        a, b, alpha = problems.setup_tree(g, 11, 5, seed=1 + rank)
        zeros = [torch.zeros((1 << l, 1 << l), dtype=torch.float64, device="cuda")
                 for l in range(g.tree_depth + 1)]
        tol, dtype = TOL, "f64" if args.precision == "fp64" else "f32+f64"

        def reset():
            for l, z in enumerate(zeros):
                a.set(z, level=l)

        def solve():
            return g.poisson(a, b, alpha=alpha, tolerance=tol)
        config = {"workload": "two_phase_tree: the two_phase_2d problem on a quadtree, level < 5 "
                              "everywhere and cells within 4 cells of r = 0.25 refined up to "
                              "level 11 (%d leaves), tolerance 1e-6, at most 100 V-cycles"
                              % g.leaves,
                  "grid": "quadtree levels 5-11", "form": args.precision,
                  "relax": "red-black Gauss-Seidel",
                  "parallelism": "replicas" if ws > 1 else "1 gpu"}
    elif args.workload == "random_field_batch":
        from basilisk_b200.autograd import Problem, solve as dsolve
        B, depth = 16, 9
        pr = Problem(2, depth, periodic=(0, 1), tolerance=1e-8, precision=args.precision,
                     lanes=args.lanes)
        g = pr.grid
        if args.lanes == 1:
            g.set_stream(torch.cuda.current_stream().cuda_stream)
        inst = [problems.random_field_2d(depth, seed=3 + rank, instance=k) for k in range(2*B)]
        dev = lambda x: torch.tensor(np.stack(x), dtype=torch.float64, device="cuda")
        kappa = dev([d["kappa"] for d in inst[:B]])
        b = dev([d["b"] for d in inst[:B]])
        b = b - b.mean(dim=(1, 2), keepdim=True)

        def face_exp(k):
            """alpha = exp(mean of the two cell kappas) on every face, periodic
            (face n is the image of face 0)"""
            kx = torch.cat([k[:, -1:], k, k[:, :1]], dim=1)
            ky = torch.cat([k[:, :, -1:], k, k[:, :, :1]], dim=2)
            return [torch.exp((kx[:, :-1] + kx[:, 1:]) / 2), torch.exp((ky[:, :, :-1] + ky[:, :, 1:]) / 2)]
        with torch.no_grad():
            a_obs = dsolve(pr, b, alpha=face_exp(dev([d["kappa"] for d in inst[B:]])))
            a_obs = a_obs - a_obs.mean(dim=(1, 2), keepdim=True)
        tol, dtype = 1e-8, "f64" if args.precision == "fp64" else "f32+f64"
        grads = {}

        def reset():
            pass

        def solve():
            k = kappa.clone().requires_grad_(True)
            a_ = dsolve(pr, b, alpha=face_exp(k))
            a_ = a_ - a_.mean(dim=(1, 2), keepdim=True)
            loss = 0.5 * ((a_ - a_obs) ** 2).sum()
            loss.backward()
            grads["kappa"] = k.grad
            st = dict(pr.stats[-1]) if pr.stats else {"i": 0, "resb": 0, "resa": 0, "nrelax": 0}
            return st
        config = {"workload": "random_field_batch: 16 independent 512^2 periodic Poisson solves, "
                              "alpha = exp(kappa) on faces (kappa a Gaussian random field, "
                              "length 0.05), b zero-mean bumps; one step = forward solves + "
                              "adjoint solves + face gradients of L = 1/2 |a - a_obs|^2 "
                              "w.r.t. kappa, tolerance 1e-8",
                  "grid": "16 x 512^2 (depth 9)", "form": args.precision,
                  "relax": "red-black Gauss-Seidel",
                  "lanes": "%d grids on their own streams, one host thread each" % args.lanes,
                  "parallelism": "replicas" if ws > 1 else "1 gpu"}
    elif args.workload == "sharded_2d":
        from basilisk_b200.shard import ShardedGrid, dims_create
        dims = dims_create(args.blocks, 2)
        if dims[0] != dims[1] or dims[0] & (dims[0] - 1):
            raise SystemExit("--blocks must give a square power-of-two arrangement (4, 16, ...)")
        prob = problems.two_phase_2d(depth=DEPTH, seed=1 + rank)
        ndev = torch.cuda.device_count()
        devices = [d % ndev for d in range(args.blocks)] if ws == 1 else [local]
        sg = ShardedGrid(2, DEPTH - int(math.log2(dims[0])), dims=dims, relax="rbgs",
                         devices=devices)
        a = sg.scalar()
        for side in range(4):
            a.bc(side, "dirichlet", 0.0)
        b = sg.scalar(prob["b"])
        alpha = sg.face_vector(prob["alpha"])
        zero = np.zeros(prob["b"].shape)
        tol, dtype = TOL, "f64"

        def reset():
            a.set(zero)

        def solve():
            return sg.poisson(a, b, alpha=alpha, tolerance=tol)
        config = {"workload": "sharded_2d: the two_phase_2d problem (2048^2, tolerance 1e-6) "
                              "decomposed into %dx%d blocks of %d^2 (grid/multigrid-mpi.h), FP64, "
                              "ghost slabs exchanged after every pass" % (dims[0], dims[1],
                                                                          2048 // dims[0]),
                  "grid": "2048x2048 as %dx%d blocks" % dims, "relax": "red-black Gauss-Seidel",
                  "devices": "%d block(s) per device on %d device(s)"
                             % (max(1, args.blocks // max(1, len(set(devices)))), len(set(devices))),
                  "parallelism": "replicas" if ws > 1 else "1 process"}
    elif args.workload == "viscosity_2d":
        depth = 11
        n = 1 << depth
        g = bmg.Grid(2, depth, relax="rbgs")
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        lv = problems.two_phase_tree_levels(depth, seed=5 + rank)[depth]
        rng = np.random.default_rng(6 + rank)
        u0 = [problems.gaussian_bumps(n, rng), problems.gaussian_bumps(n, rng)]
        # face viscosity 1/100 of the face density: mu and rho ratios 1000
        ax, ay = problems.two_phase_alpha(n)
        mu = g.face_vector([0.01 / ax, 0.01 / ay])
        x, y = problems.centers(2, n)
        f = 0.5 * (1.0 - np.tanh((np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2) - 0.25) * n / 2.0))
        rho = g.scalar(f * (1.0 - 1000.0) + 1000.0)
        uu = g.vector()
        for c in uu:
            for side in range(4):
                c.bc(side, "dirichlet", 0.0)
        dev = [torch.tensor(c, dtype=torch.float64, device="cuda") for c in u0]
        tol, dtype = TOL, "f64"
        bmg.set_tolerance(tol)      # viscosity () solves to the global TOLERANCE
        del lv

        def reset():
            for c, d in zip(uu, dev):
                c.set(d)

        def solve():
            return g.viscosity(uu, mu, rho, 1e-3)
        config = {"workload": "viscosity_2d: implicit viscous step of a 2048^2 velocity field "
                              "(two components, Gaussian bumps), rho two-phase (ratio 1000), "
                              "face mu = 0.01 rho_face (ratio 1000), dt = 1e-3, no-slip walls, "
                              "TOLERANCE 1e-6",
                  "grid": "2048x2048 (depth 11)", "relax": "red-black (colour-buffered)",
                  "parallelism": "replicas" if ws > 1 else "1 gpu"}
    else:
        prob = problems.helmholtz_3d(depth=8, seed=2 + rank)
        g = bmg.Grid(3, 8, relax="rbgs", precision=args.precision)
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        a, b, alpha, lam = problems.setup(g, prob)
        zero = torch.zeros(prob["b"].shape, dtype=torch.float64, device="cuda")
        tol, dtype = prob["tolerance"], "f64" if args.precision == "fp64" else "f32+f64"

        def reset():
            a.set(zero)

        def solve():
            return g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=tol)
        config = {"workload": "helmholtz_3d: 256^3 periodic Helmholtz, alpha = 1e-2 stored on "
                              "every face, lambda = -1000, b ~ N(0,1) smoothed, tolerance %g"
                              % tol,
                  "grid": "256^3 (depth 8)", "form": args.precision,
                  "relax": "red-black Gauss-Seidel",
                  "parallelism": "replicas" if ws > 1 else "1 gpu"}
    if args.workload == "random_field_batch":
        grids = [ln.grid for ln in pr.lanes]
    elif args.workload == "sharded_2d":
        grids = sg.blocks
    else:
        grids = [g]
    for gg in grids:
        gg.set_timing(True)
    clocks.start()
    for _ in range(args.warmup):
        reset()
        solve()
    torch.cuda.synchronize()
    barrier(ws)
    for gg in grids:
        gg.reset_counters()
    times, st = [], None
    t_begin = time.monotonic()
    for _ in range(args.steps):
        flush_l2(flush)
        reset()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = solve()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks.window(t_begin, time.monotonic())
    clk = clocks.stop()
    barrier(ws)
    cs = [gg.counters() for gg in grids]
    c = {k: sum(x[k] for x in cs) for k in cs[0]}
    ms = max_over_ranks(ws, sum(times) / len(times))
    if rank != 0:
        return
    unit = "gradient steps/s (16 instances each)" if args.workload == "random_field_batch" \
        else "solves/s"
    line = {"metric": "time-to-residual, %s" % args.workload, "value": ws * 1e3 / ms,
            "unit": unit, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype, "data": "synthetic", "config": config,
            "mgstats": {k: st[k] for k in ("i", "resb", "resa", "nrelax")},
            "vcycle": {"cycles": c["cycles"], "ms_per_cycle": c["cycle_ms"] / max(1, c["cycles"]),
                       "launches_per_cycle": c["launches"] / max(1, c["cycles"]),
                       "vcycle_gbs": c["bytes"] / (c["cycle_ms"] * 1e-3) / 1e9
                       if c["cycle_ms"] and c["bytes"] else None},
            "clocks": clk, "gpu_launches": int(c["launches"])}
    # the whole step's algorithmic bytes (every V-cycle kernel, each array
    # pass once at its storage precision; on the tree plus 4 B per list
    # index) over its device time
    peak, peak_kind = load_peaks()
    if c["bytes"]:
        ach = c["bytes"] / args.steps / (ms * 1e-3) / 1e9
        line["roofline"] = {"bound": "hbm", "kernel": "whole step (all V-cycle kernels)",
                            "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                            "traffic": None, "peak_kind": peak_kind,
                            "note": "algorithmic bytes of the step over its CUDA-event time; "
                                    "no ncu capture of this workload, so no DRAM traffic"}
    if not args.no_cpu and args.workload == "helmholtz_3d":
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle import oracle
        from helpers import oracle_grid
        threads = os.cpu_count()
        o = oracle_grid(prob, relax=oracle.RELAX_GS, threads=threads)
        t0 = time.perf_counter()
        cst = o.poisson(tolerance=tol)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": threads,
                                "kind": "port",
                                "sample": "1 full solve of the same problem (%d V-cycles), "
                                          "lexicographic GS, %d OpenMP threads" % (cst["i"], threads)}
    if not args.no_cpu and args.workload == "random_field_batch":
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle import oracle
        threads = os.cpu_count()
        kq = [d["kappa"] for d in inst[:2]]
        bq = b[:2].cpu().numpy()
        obs = a_obs[:2].cpu().numpy()
        n = 1 << depth
        t_cpu = 0.0
        for k in range(2):
            kk = np.asarray(kq[k])
            kx = np.concatenate([kk[-1:], kk, kk[:1]], axis=0)
            ky = np.concatenate([kk[:, -1:], kk, kk[:, :1]], axis=1)
            alpha = [np.exp((kx[:-1] + kx[1:]) / 2), np.exp((ky[:, :-1] + ky[:, 1:]) / 2)]
            for rhs_kind in ("forward", "adjoint"):
                o = oracle.Grid(2, depth, relax=oracle.RELAX_GS, threads=threads)
                o.set_periodic(0); o.set_periodic(1)
                o.set_alpha(alpha)
                o.set_lambda_const(0.0)
                if rhs_kind == "forward":
                    rhs = bq[k]
                else:
                    rhs = a_fwd - obs[k]
                    rhs = rhs - rhs.mean()
                o.set_b(rhs)
                o.set_a(np.zeros((n, n)))
                t0 = time.perf_counter()
                o.poisson(tolerance=tol)
                t_cpu += time.perf_counter() - t0
                if rhs_kind == "forward":
                    a_fwd = o.get_a() - o.get_a().mean()
        step = t_cpu * B / 2
        line["cpu_baseline"] = {"value": 1.0 / step, "unit": unit, "cores": threads,
                                "kind": "port",
                                "sample": "the forward and adjoint solves of 2 of the 16 "
                                          "instances (lexicographic GS, %d OpenMP threads, %.1f s), "
                                          "scaled to 16; the face gradients are not timed"
                                          % (threads, t_cpu)}
    if not args.no_cpu and args.workload == "viscosity_2d":
        # the oracle's viscosity () (viscosity.h:169-183 restated, the
        # reference's lexicographic GS relax_viscosity) on the same fields
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle import oracle
        threads = os.cpu_count()
        o = oracle.Grid(2, depth, relax=oracle.RELAX_GS, threads=threads)
        for comp in range(2):
            for side in range(4):
                o.set_visc_bc(comp, side, oracle.DIRICHLET, 0.0)
        o.set_u(u0)
        o.set_mu([0.01 / ax, 0.01 / ay])
        o.set_rho(f * (1.0 - 1000.0) + 1000.0)
        oracle.set_globals(2, tolerance=tol)
        try:
            t0 = time.perf_counter()
            cst = o.viscosity(dt=1e-3)
            dt_cpu = time.perf_counter() - t0
        finally:
            oracle.set_globals(2, tolerance=1e-3)
        line["cpu_baseline"] = {"value": 1.0 / dt_cpu, "unit": "solves/s", "cores": threads,
                                "kind": "port",
                                "sample": "1 viscous step of the same fields (%d V-cycles), "
                                          "lexicographic GS, %d OpenMP threads" % (cst["i"], threads)}
    if not args.no_cpu and args.workload == "sharded_2d":
        # the reference's MPI multigrid runs this decomposition on 2x2 ranks;
        # its CPU restatement here is the single-domain oracle with the same
        # coarsest level (a block's level 1 is the domain's level 1 + log2 dims)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle import oracle
        from helpers import oracle_grid
        threads = os.cpu_count()
        o = oracle_grid(prob, relax=oracle.RELAX_GS, threads=threads)
        t0 = time.perf_counter()
        cst = o.poisson(tolerance=tol, minlevel=1 + int(math.log2(dims[0])))
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": threads,
                                "kind": "port",
                                "sample": "1 full solve of the same problem on one domain with the "
                                          "blocks' coarsest level (%d V-cycles), lexicographic GS, "
                                          "%d OpenMP threads" % (cst["i"], threads)}
    if not args.no_cpu and args.workload == "two_phase_tree":
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle import tree as otree
        import golden_drivers as gd
        # the error of this form's solution (tolerance 1e-6) against the tree
        # oracle (red-black, FP64) driven to 1e-9 on the same tree
        tf = otree.Tree(11, 1.0, (0.0, 0.0))
        tf.set_relax(otree.RELAX_RBGS)
        tf.refine(problems.band_refinement(11, 5))
        gd.two_phase_tree(tf, seed=1)
        otree.set_niter(nitermax=300)
        try:
            fst = tf.poisson(tolerance=1e-9, nrelax=4, minlevel=1)
        finally:
            otree.set_niter(nitermax=100)
        dev_a, ref_a = [], []
        for l in range(tf.depth + 1):
            leaf = (tf.flags(l) & otree.LEAF) != 0
            ref_a.append(tf.get_level(otree.A, l)[leaf])
            dev_a.append(a.get(level=l)[leaf])
        ref_a, dev_a = np.concatenate(ref_a), np.concatenate(dev_a)
        line["error_vs_oracle"] = {
            args.precision: float(np.abs(dev_a - ref_a).max() / np.abs(ref_a).max()),
            "oracle_residual": fst["resa"], "oracle_cycles": fst["i"],
            "note": "max over leaves |a - a_oracle| / max |a_oracle|, this form at residual "
                    "1e-6, the tree oracle (red-black, FP64) driven to 1e-9"}
        t = otree.Tree(11, 1.0, (0.0, 0.0))
        t.set_relax(otree.RELAX_GS)
        t.refine(problems.band_refinement(11, 5))
        gd.two_phase_tree(t, seed=1)
        t0 = time.perf_counter()
        cst = t.poisson(tolerance=TOL, nrelax=4, minlevel=1)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": 1, "kind": "port",
                                "sample": "1 full solve of the same tree (%d V-cycles), the "
                                          "reference's traversal-order Gauss-Seidel, 1 thread"
                                          % cst["i"]}
    print(json.dumps(line), flush=True)


def run_reference(args, ws, rank):
    """The reference arm: the CPU implementation, full solves of the same
    workload, on rank 0 only."""
    from basilisk_b200 import problems
    if rank != 0:
        return
    prob = problems.two_phase_2d(depth=DEPTH, seed=1)
    budget = float(os.environ.get("BMG_CPU_BUDGET", "90"))
    times, st, threads = [], None, None
    for _ in range(max(1, args.steps)):
        t, st, threads = cpu_solve(prob)
        times.append(t)
        if sum(times) > budget:
            break
    ms = 1e3 * sum(times) / len(times)
    val = 1e3 / ms
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": len(times), "warmup": 0, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "two_phase_2d 2048^2 variable-coefficient Poisson, density "
                                   "ratio 1000, b ~ N(0,1), Dirichlet 0, tolerance 1e-6",
                       "grid": "2048x2048 (depth 11)", "parallelism": "cpu-openmp"},
            "mgstats": {k: st[k] for k in ("i", "resb", "resa", "nrelax")},
            "cpu_baseline": {"value": val, "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": "%d full solve(s) of the same workload, lexicographic GS, "
                                       "%d OpenMP threads" % (len(times), threads)},
            "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bmg", choices=["bmg", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline solve")
    ap.add_argument("--profile", choices=["fp64", "mixed"], default=None,
                    help="profiling run: only this form, no e2e, no CPU baseline, no JSON")
    ap.add_argument("--depth", type=int, default=DEPTH, help="grid depth (profiling runs)")
    ap.add_argument("--workload", choices=["two_phase_2d", "two_phase_tree", "helmholtz_3d",
                                           "random_field_batch", "viscosity_2d", "sharded_2d"],
                    default="two_phase_2d",
                    help="two_phase_2d: the headline; the others print their own line")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="form of the helmholtz_3d and random_field_batch workloads")
    ap.add_argument("--blocks", type=int, default=4,
                    help="sharded_2d: number of blocks (a square power-of-two arrangement)")
    ap.add_argument("--lanes", type=int, default=8,
                    help="random_field_batch: grids solving instances concurrently")
    args = ap.parse_args()
    ws, rank, local = dist_init()
    if args.impl == "bmg" and args.workload != "two_phase_2d":
        run_workload(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    from basilisk_b200 import problems
    peak, peak_kind = load_peaks()
    prob = problems.two_phase_2d(depth=args.depth if args.profile else DEPTH, seed=1 + rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    if args.profile:
        s = Solver(prob, args.profile)
        t, st, c = time_steps(s, args.steps, args.warmup, ws, flush)
        print("profile run: %s depth %d: %.3f ms/solve, %d cycles, nrelax %d, %d launches"
              % (args.profile, prob["depth"], sum(t) / len(t), st["i"], st["nrelax"],
                 c["launches"]), flush=True)
        return

    # plain FP64 form
    s64 = Solver(prob, "fp64")
    t64, st64, c64 = time_steps(s64, args.steps, args.warmup, ws, flush)
    a64 = s64.a.get()
    # mixed form (headline), with clocks sampled during its timed region
    smx = Solver(prob, "mixed")
    clocks = ClockSampler(local)
    clocks.start()
    tmx, stmx, cmx = time_steps(smx, args.steps, args.warmup, ws, flush, clocks)
    clk = clocks.stop()
    amx = smx.a.get()

    ms_mx = max_over_ranks(ws, sum(tmx) / len(tmx))
    ms_64 = max_over_ranks(ws, sum(t64) / len(t64))
    err = float(np.abs(amx - a64).max() / np.abs(a64).max())

    # e2e through the public API with host buffers (mixed form)
    te2e, h2d, d2h = e2e_steps(prob, args.steps, max(1, args.warmup // 2), "mixed")
    ms_e2e = max_over_ranks(ws, sum(te2e) / len(te2e))

    if rank != 0:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    def cyc(c):
        return {"cycles": c["cycles"], "sweeps": c["sweeps"],
                "vcycle_gbs": c["bytes"] / (c["cycle_ms"] * 1e-3) / 1e9 if c["cycle_ms"] else None,
                "relax_gbs": c["relax_bytes"] / (c["relax_ms"] * 1e-3) / 1e9 if c["relax_ms"] else None,
                "bytes_per_cycle": c["bytes"] / max(1, c["cycles"]),
                "ms_per_cycle": c["cycle_ms"] / max(1, c["cycles"])}

    f64, fmx = cyc(c64), cyc(cmx)
    relax_avg_ms = cmx["relax_ms"] / max(1, cmx["relax_sweeps"])
    relax_bytes = cmx["relax_bytes"] / max(1, cmx["relax_sweeps"])
    achieved = relax_bytes / (relax_avg_ms * 1e-3) / 1e9 if relax_avg_ms else None
    # the DRAM rate of the same kernel: its measured traffic per launch of
    # four sweeps over the time of four sweeps
    dram = TILE_LAUNCH_DRAM_BYTES / (4 * relax_avg_ms * 1e-3) / 1e9 if relax_avg_ms else None
    line = {
        "metric": METRIC, "value": ws * 1e3 / ms_mx, "unit": "solves/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mx,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": {"workload": "two_phase_2d 2048^2 variable-coefficient Poisson, density ratio "
                               "1000, b ~ N(0,1), Dirichlet 0, tolerance 1e-6",
                   "grid": "2048x2048 (depth 11)", "form": "mixed FP32 cycles + FP64 refinement",
                   "relax": "red-black Gauss-Seidel", "parallelism": "replicas" if ws > 1 else "1 gpu",
                   "l2": "flushed (256 MB write) before every timed step; inputs > L2"},
        "time_to_residual_ms": {"mixed": ms_mx, "fp64": ms_64, "speedup_mixed_vs_fp64": ms_64 / ms_mx},
        "mgstats": {"mixed": {k: stmx[k] for k in ("i", "resb", "resa", "nrelax")},
                    "fp64": {k: st64[k] for k in ("i", "resb", "resa", "nrelax")}},
        "mixed_vs_fp64_rel_error": err,
        "vcycle": {"mixed": fmx, "fp64": f64},
        "roofline": {"bound": "hbm",
                     "kernel": "k_relax_tile2d_w (finest level, 4 red-black sweeps per launch)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None,
                     # DRAM bytes (read + write) of one finest-level launch of four
                     # sweeps, from an ncu capture of that kernel; the algorithmic
                     # bytes of that launch are 335.5e6
                     "traffic": TILE_LAUNCH_DRAM_BYTES, "traffic_per": "launch (4 sweeps)",
                     "peak_kind": peak_kind,
                     "note": "achieved counts algorithmic bytes (5 arrays per cell per sweep); "
                             "with 4 sweeps per launch on on-chip tiles the DRAM traffic is "
                             "lower, so the DRAM rate (dram_achieved) is the HBM utilisation "
                             "and vcycle_frac the whole V-cycle's algorithmic rate",
                     "dram_achieved": dram, "dram_frac": dram / peak if dram else None,
                     "vcycle_frac": {"mixed": fmx["vcycle_gbs"] / peak if fmx["vcycle_gbs"] else None,
                                     "fp64": f64["vcycle_gbs"] / peak if f64["vcycle_gbs"] else None}},
        "clocks": clk,
        "gpu_launches": int(cmx["launches"]),
        "e2e": {"value": ws * 1e3 / ms_e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
    }
    if not args.no_cpu:
        try:
            af, fres, a9 = oracle_floor(prob)
            rel = lambda x: float(np.abs(x - af).max() / np.abs(af).max())
            line["error_vs_oracle"] = {
                "fp64": rel(a64), "mixed": rel(amx), "oracle_floor": fres,
                "oracle_1e-9_vs_floor": rel(a9),
                "note": "max |a - a_oracle| / max |a_oracle|, both forms at residual 1e-6, "
                        "the oracle (red-black, FP64) driven to its residual floor"}
        except Exception as e:  # reported, never required
            line["error_vs_oracle"] = {"fp64": None, "mixed": None, "oracle_floor": None,
                                       "note": "failed: %s" % e}
        try:
            t, st, threads = cpu_solve(prob)
            line["cpu_baseline"] = {
                "value": 1.0 / t, "unit": "solves/s", "cores": threads, "kind": "port",
                "sample": "1 full solve of the same workload (%d V-cycles, final nrelax %d), "
                          "lexicographic GS, %d OpenMP threads" % (st["i"], st["nrelax"], threads)}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": 0, "kind": "port",
                                    "sample": "failed: %s" % e}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
