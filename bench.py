"""Benchmark: the IPM numeric core on the 2D SIMP compliance KKT (128 x 64).

One step = one interior-point iteration's numeric core on the full-space 2D
SIMP KKT system (n = 58,504, nnz = 2.24e6), all on the GPU:
  Hessian of the Lagrangian scattered into the CSR KKT values, barrier
  diagonal + delta_w added, multifrontal LDL^T factorization with the
  inertia read back, condensed residual, solve, one iterative-refinement
  step (K p, residual, correction solve), bound-dual back-substitution,
  fraction-to-boundary step length, step application, gradient.
`value` is the KKT factorization throughput in TFLOP/s: the algorithmic
factor flops of the step (sum over fronts of p^3/3 + p^2 c + p c^2) divided
by the device time of the whole step.  `e2e` is the same metric through the
public SparseLDL API with the KKT values and right-hand side starting in
host memory and the solution copied back every step.

Extra fields of the same JSON line (1 GPU): `simp3d_factor` (3D SIMP
cantilever 48x24x24 KKT: FP64 factor + solve, and the mixed-precision form
with FP32 fronts, tensor-core Schur updates and FP64 refinement),
`ipm_solve` (the cart-pole N = 100 problem solved end to end, p50/p99, with
the same driver over the reference's host core beside it), `batch_solve`
(512 cart-pole problems solved together, FP64 and mixed, with the
single-problem device path beside it), `serve` (a Poisson request stream at
80% of the serving loop's measured capacity, continuous batching,
p50/p95/p99 latency).  `--no-3d`, `--no-ipm-solve`, `--batch 0`,
`--serve-requests 0` skip them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank runs an independent replica on its own GPU
(the path does not shard); the device time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("IPM solves/s & KKT factor TFLOP/s, mixed vs FP64 GPU at 1e-8 err; "
          "p50/p99 latency")
WORKLOAD = "2D SIMP compliance 128x64 full-space KKT, one IPM iteration core"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--solves", type=int, default=5)
    ap.add_argument("--no-ipm-solve", action="store_true")
    ap.add_argument("--batch", type=int, default=512,
                    help="instances in the batched cart-pole solve (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=600,
                    help="requests in the serving run (0: skip)")
    ap.add_argument("--clock-dir", default=tempfile.gettempdir(),
                    help="folder for the nvidia-smi clock samples of the timed region")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default panel forms and solve schedule of the "
                         "2D KKT instead of the autotuner's")
    ap.add_argument("--no-3d", action="store_true",
                    help="skip the 3D SIMP 48x24x24 factorization")
    ap.add_argument("--simp3d", default="48,24,24",
                    help="mesh of the 3D SIMP factorization, NX,NY,NZ (a smaller "
                         "mesh for profiling)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(values, device=None):
    """Element-wise maximum of a list of floats over all ranks (device times
    are reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def sum_over_ranks(values, device=None):
    """Element-wise sum of a list of floats over all ranks (work counts of
    the replicas)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()]


def relaunch_under_torchrun(args):
    """`python bench.py --gpus N` (N > 1) outside torchrun: start N ranks on
    this node with torch.distributed.run (replicas, one per GPU)."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(args.gpus), "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    os.execv(sys.executable, cmd)


def shard(items, rank, world):
    """This rank's contiguous share of a list of independent problems."""
    b0, b1 = replica_items(len(items), rank, world)
    return items[b0:b1]


def replica_items(n_items, rank, world):
    """Independent problems are split over ranks in contiguous blocks (the
    replicas-only decomposition): returns this rank's [begin, end)."""
    base, extra = divmod(n_items, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def config(args, world):
    return {"workload": WORKLOAD, "n": None, "nnz": None,
            "mesh": "%dx%d" % (args.nx, args.ny), "ordering": "AMD",
            "precision": "fp64", "parallelism": "replicas%d" % world,
            "l2": "256 MiB buffer written between timed steps"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, path, index):
        self.path = path
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines()]
            sm = [float(r[0]) for r in rows if r[0].strip().isdigit()]
            mx = max(float(r[1]) for r in rows)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                     "sw_power_cap"]
            reasons = sorted({names[k] for r in rows for k in range(4)
                              if r[4 + k].strip() == "Active"})
            return {"sm_mhz": float(np.median(sm)) if sm else None,
                    "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0}


# --------------------------------------------------------------- our arm
class Core:
    """The IPM iteration numeric core on one GPU (see module docstring)."""

    def __init__(self, device, nx, ny):
        import torch
        from amigo_b200 import linalg
        from amigo_b200.fem import Simp2DDevice
        from amigo_b200.ipm import InteriorPointOptimizer
        from amigo_b200.problems.simp2d import Simp2D
        self.torch = torch
        self.dev = device
        m = Simp2D(nx, ny)
        self.m = m
        self.fem = Simp2DDevice(m, device)
        self.K = linalg.CSRMat(m.n, m.n, m.rowp, m.cols, device=device)
        self.ldl = linalg.SparseLDL(self.K, ustab=0.01, pivot_tol=1e-14,
                                    order=linalg.OrderingType.AMD)
        self.opt = InteriorPointOptimizer(m.mult, m.lower, m.upper, device=device)
        self.opt.relax_bounds()
        f64 = dict(dtype=torch.float64, device=device)
        self.x = torch.from_numpy(m.initial_point()).to(device)
        self.vars = self.opt.create_opt_vector(self.x)
        self.opt.initialize_multipliers_and_slacks(0.1, None, self.vars)
        self.grad = torch.zeros(m.n, **f64)
        self.res = torch.zeros(m.n, **f64)
        self.diag = torch.zeros(m.n, **f64)
        self.px = torch.zeros(m.n, **f64)
        self.r2 = torch.zeros(m.n, **f64)
        self.kp = torch.zeros(m.n, **f64)
        self.upd = self.opt.create_opt_vector()
        self.tmp = self.opt.create_opt_vector()
        self.primal = torch.from_numpy(~m.mult).to(device)
        self.mu = 0.1
        self.fem.gradient(self.x, 1.0, self.grad)
        self.flops = None
        self.launches = None

    def step(self):
        torch = self.torch
        m, opt, v = self.m, self.opt, self.vars
        self.fem.hessian(v.x, 1.0, self.K.vals)
        opt.compute_diagonal(v, self.diag)
        self.diag.add_(self.primal, alpha=1e-8)
        self.K.add_diagonal(self.diag)
        self.ldl.factor()
        inertia = self.ldl.get_inertia()
        opt.compute_residual(self.mu, v, self.grad, self.res)
        self.px.copy_(self.res)
        self.ldl.solve_device(self.px)
        # one refinement step on the condensed system
        self.K.mult(self.px, self.kp)
        torch.sub(self.res, self.kp, out=self.r2)
        self.ldl.solve_device(self.r2)
        self.px.add_(self.r2)
        opt.compute_update(self.mu, v, self.px, self.upd)
        ax, xi, az, zi = opt.compute_max_step(0.99, v, self.upd)
        opt.apply_step_update(ax, az, v, self.upd, self.tmp)
        self.fem.gradient(self.tmp.x, 1.0, self.grad)
        return inertia


def run_ours(args, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    core = Core(device, args.nx, args.ny)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
    tuning = None
    for w in range(args.warmup):
        inertia = core.step()
        if w == 0 and not args.no_autotune:
            # panel forms and solve schedule picked by timing them on this
            # KKT (ab_ldl_autotune); the remaining warm-up steps use them
            try:
                tuning = core.ldl.autotune(reps=3)
            except Exception as e:   # the defaults stay on the handle
                tuning = {"error": str(e)[:200]}
    torch.cuda.synchronize()
    npiv_ours, _ = core.ldl.node_pivots()
    st = core.ldl.stats()
    flops = st["flops"]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    fev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    sev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    from amigo_b200 import _lib
    launches0 = _lib.lib().ab_launch_count()
    clk = ClockSampler(os.path.join(args.clock_dir, "clocks_rank%d.csv" % rank), local)
    t0 = time.time()
    with clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            # factor timing inside the step (same stream)
            core.fem.hessian(core.vars.x, 1.0, core.K.vals)
            core.opt.compute_diagonal(core.vars, core.diag)
            core.diag.add_(core.primal, alpha=1e-8)
            core.K.add_diagonal(core.diag)
            fev[k][0].record(stream)
            core.ldl.factor()
            fev[k][1].record(stream)
            core.ldl.get_inertia()
            opt, v = core.opt, core.vars
            opt.compute_residual(core.mu, v, core.grad, core.res)
            core.px.copy_(core.res)
            sev[k][0].record(stream)
            core.ldl.solve_device(core.px)
            core.K.mult(core.px, core.kp)
            torch.sub(core.res, core.kp, out=core.r2)
            core.ldl.solve_device(core.r2)
            sev[k][1].record(stream)
            core.px.add_(core.r2)
            opt.compute_update(core.mu, v, core.px, core.upd)
            ax, xi, az, zi = opt.compute_max_step(0.99, v, core.upd)
            opt.apply_step_update(ax, az, v, core.upd, core.tmp)
            core.fem.gradient(core.tmp.x, 1.0, core.grad)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    wall = time.time() - t0
    launches = _lib.lib().ab_launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    fac_ms = [a.elapsed_time(b) for a, b in fev]
    sol_ms = [a.elapsed_time(b) for a, b in sev]
    dev_ms = float(np.sum(step_ms))
    fac_tot = float(np.sum(fac_ms))
    dev_ms, fac_tot = max_over_ranks([dev_ms, fac_tot], device)
    value = world * flops * args.steps / (dev_ms * 1e-3) / 1e12

    # e2e through the public API with host buffers
    e2e = run_e2e(core, args, device)
    try:
        graph = solve_graph_bench(core)
    except Exception as e:
        graph = {"error": str(e)[:200]}

    out = {
        "metric": METRIC,
        "value": round(value, 6),
        "unit": "TFLOP/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dev_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: 2D SIMP KKT at the seeded initial point",
        "config": dict(config(args, world), n=core.m.n, nnz=core.m.nnz),
        "factor_flops_per_step": flops,
        "factor_ms_per_step": round(fac_tot / args.steps, 4),
        "ipm_iterations_per_s": round(world * args.steps / (dev_ms * 1e-3), 3),
        "wall_s": round(wall, 3),
        "e2e": e2e,
        "gpu_launches": int(launches),
        "solve_ms_per_step": round(float(np.sum(sol_ms)) / args.steps, 4),
        "clocks": clk.summary(),
        "ldl_stats": st,
        "inertia": [int(inertia[0]), int(inertia[1])],
        "threads": threads_env(),
        "autotune": tuning,
        "solve_graph": graph,
    }
    core_npiv = npiv_ours
    out["roofline"] = roofline(core, fac_tot / args.steps)
    out["_npiv"] = core_npiv
    if not args.no_3d:
        # one factorization per GPU: every replica runs it on its own device
        del core, flush
        torch.cuda.empty_cache()
        out["simp3d_factor"] = simp3d_bench(
            device, dims=tuple(int(v) for v in args.simp3d.split(",")))
        torch.cuda.empty_cache()
    if not args.no_ipm_solve:
        out["ipm_solve"] = ipm_solve_bench(device, args.solves)
        if args.batch > 0:
            out["batch_solve"] = batch_solve_bench(device, args.batch, rank=rank,
                                                   world=world)
            if args.serve_requests > 0:
                cap = out["batch_solve"]["solves_per_s"] / world
                out["serve"] = serve_bench(device, args.serve_requests, cap,
                                           rank=rank, world=world)
    return out


def barrier(device):
    import torch
    import torch.distributed as dist
    torch.cuda.synchronize(device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def serve_bench(device, n_requests, batch_capacity, rank=0, world=1):
    """Serving: a stream of cart-pole solve requests (N ~ U{50..400}) with
    Poisson arrivals at 80% of the serving loop's own capacity, continuous
    batching (serve.Server: admission at iteration boundaries by slots and a
    150 GB device-memory budget from symbolic workspace estimates).  The
    capacity is measured first with 256 requests that all arrive at once."""
    from amigo_b200 import serve
    _, sat = serve.Server(device, mem_budget=150e9, max_batch=512).run(
        serve.make_stream(256, rate=1e6, seed=12), time_limit=120)
    capacity = sat["solves_per_s"]
    rate = 0.8 * capacity
    # replicas: rank r serves its contiguous share of the request stream
    # (each GPU its own queue and memory budget), at its share of the rate
    b0, b1 = replica_items(n_requests, rank, world)
    reqs = serve.make_stream(n_requests, rate * world, seed=11)[b0:b1]
    srv = serve.Server(device, mem_budget=150e9, max_batch=512)
    barrier(device)
    _, summ = srv.run(reqs, time_limit=240)
    if world > 1:
        # whole-job throughput; latency percentiles are the slowest rank's
        summ["solves_per_s"], = sum_over_ranks([summ["solves_per_s"]], device)
        for key in ("p50_ms", "p95_ms", "p99_ms"):
            if key in summ:
                summ[key], = max_over_ranks([summ[key]], device)
        summ["replicas"] = world
    summ = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in summ.items()}
    summ.update(arrival_rate_per_s=round(rate, 3),
                serving_capacity_per_s=round(capacity, 3),
                batched_capacity_per_s=batch_capacity,
                mix="cart-pole requests only (the 70% class of the serving mix)")
    return summ


def simp3d_bench(device, reps=2, dims=(48, 24, 24)):
    """The 3D SIMP cantilever 48x24x24 KKT (n = 272,650, nnz = 4.1e7; AMD;
    largest front ~25k): one FP64 factorization and one solve per rep,
    CUDA events, after one warm-up factorization.  Diagonal: 1e-2 + U(0, 1)
    on the primal rows (quasi-definite), so the inertia is known:
    (primal + fixed multipliers, multipliers - fixed multipliers)."""
    import torch
    from amigo_b200 import linalg
    from amigo_b200.problems.simp3d import Simp3D
    t0 = time.perf_counter()
    m = Simp3D(*dims)
    dm = m.device_model(device)
    K = linalg.CSRMat(m.n, m.n, m.rowp, m.cols, device=device)
    ldl = linalg.SparseLDL(K, order=linalg.OrderingType.AMD)
    setup_s = time.perf_counter() - t0
    x = torch.from_numpy(m.initial_point()).to(device)
    dm.hessian(x, 1.0, K.vals)
    g = torch.Generator(device=device).manual_seed(0)
    prim = torch.from_numpy(~m.mult).to(device)
    d = torch.where(prim, 1e-2 + torch.rand(m.n, dtype=torch.float64,
                                            device=device, generator=g), 0.0)
    d[torch.from_numpy(m.fixed).long().to(device)] = 0.0
    K.add_diagonal(d)
    nfl = int(np.sum(m.mult[m.fixed]))
    want = (int((~m.mult).sum()) + nfl, int(m.mult.sum()) - nfl)
    ldl.factor()
    b = torch.randn(m.n, dtype=torch.float64, device=device, generator=g)
    stream = torch.cuda.current_stream()
    fac, sol = [], []
    for _ in range(reps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        xs = b.clone()
        e[0].record(stream)
        ldl.factor()
        e[1].record(stream)
        ldl.solve_device(xs)
        e[2].record(stream)
        torch.cuda.synchronize()
        fac.append(e[0].elapsed_time(e[1]))
        sol.append(e[1].elapsed_time(e[2]))
    kx = torch.zeros_like(xs)
    K.mult(xs, kx)
    res = (kx - b).abs().max().item()
    # normwise relative residual ||Kx - b|| / (||K|| ||x|| + ||b||), inf-norms
    rows = torch.repeat_interleave(
        torch.arange(m.n, device=device),
        torch.from_numpy(np.diff(m.rowp).astype(np.int64)).to(device))
    kinf = torch.zeros(m.n, dtype=torch.float64, device=device).index_add_(
        0, rows, K.vals.abs()).max().item()
    relres = lambda x, r: r / (kinf * x.abs().max().item() + b.abs().max().item())
    rel64 = relres(xs, res)
    st = ldl.stats()
    inertia = list(ldl.get_inertia())
    fac_s = float(np.median(fac)) * 1e-3
    # mixed precision: FP32 fronts, tensor-core Schur updates, FP64
    # refinement of the solve against the FP64 matrix
    ldl.set_precision("fp32")
    ldl.factor()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    xm = b.clone()
    r = torch.empty_like(b)
    e[0].record(stream)
    ldl.factor()
    e[1].record(stream)
    ldl.solve_device(xm)
    # refinement against the FP64 matrix until the normwise relative
    # residual is <= 1e-10 or stops improving by 2x (at most 10 steps)
    steps, prev = 0, float("inf")
    xinf = xm.abs().max().item()
    for _ in range(10):
        K.mult(xm, r)
        r.sub_(b).neg_()
        rr = r.abs().max().item() / (kinf * xinf + b.abs().max().item())
        if rr <= 1e-10 or rr > 0.5 * prev:
            break
        prev = rr
        ldl.solve_device(r)
        xm.add_(r)
        xinf = xm.abs().max().item()
        steps += 1
    e[2].record(stream)
    torch.cuda.synchronize()
    K.mult(xm, kx)
    res_m = (kx - b).abs().max().item()
    inertia_m = list(ldl.get_inertia())
    mixed = {"factor_s": round(e[0].elapsed_time(e[1]) * 1e-3, 4),
             "solve_refine_s": round(e[1].elapsed_time(e[2]) * 1e-3, 4),
             "refinement_steps": steps,
             "inertia": inertia_m,
             "inertia_equals_expected": inertia_m == list(want),
             "residual_inf": res_m,
             "relative_residual": relres(xm, res_m),
             "note": "FP32 fronts, 3xTF32 tcgen05 Schur updates, FP64 "
                     "refinement to 1e-10 or until it stalls; the mixed-"
                     "precision IPM drivers refactor in FP64 when the inertia "
                     "differs from the expected one or refinement stalls "
                     "above 1e-10"}
    return {"workload": "3D SIMP cantilever %dx%dx%d full-space KKT, FP64 "
                        "factor + solve" % tuple(dims),
            "n": int(m.n), "nnz": int(m.nnz), "flops": st["flops"],
            "factor_s": round(fac_s, 4), "solve_s": round(float(np.median(sol)) * 1e-3, 4),
            "tflops": round(st["flops"] / fac_s / 1e12, 3),
            "inertia": inertia, "inertia_expected": list(want),
            "residual_inf": res, "relative_residual": rel64,
            "max_front": st["max_front"],
            "num_delayed": st["num_delayed"], "factor_entries": st["factor_entries"],
            "host_setup_s": round(setup_s, 2), "reps": reps, "mixed": mixed}


def batch_solve_bench(device, k, sequential_sample=8, rank=0, world=1):
    """The batched-trajectories config: k cart-pole instances (N ~
    U{50..400}, pole mass ~ U(0.1, 0.5), final position ~ U(-1, 1), seed 0)
    solved together, one launch per IPM phase over all instances; beside it
    the same instances solved one after another by the single-problem
    device path (a sample of `sequential_sample`, extrapolated)."""
    import torch
    from amigo_b200 import ipm_driver
    from amigo_b200.problems.cartpole import batch_config
    from amigo_b200.problems.cartpole import CartPoleBatch
    ipm_driver.solve_batch(batch_config(k=4, seed=1), device)   # warm-up
    full = batch_config(k=k, seed=0)
    B = full if world == 1 else CartPoleBatch(shard(full.inst, rank, world))
    barrier(device)
    t = time.perf_counter()
    r = ipm_driver.solve_batch(B, device)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    barrier(device)
    t = time.perf_counter()
    rm = ipm_driver.solve_batch(B, device, precision="fp32")
    torch.cuda.synchronize()
    wall_m = time.perf_counter() - t
    wall, wall_m = max_over_ranks([wall, wall_m], device)
    conv_all, conv_m_all = sum_over_ranks([int(r["converged"].sum()),
                                           int(rm["converged"].sum())], device)
    same = rm["converged"] & r["converged"]
    obj_dev = (float(np.max(np.abs(rm["objective"][same] - r["objective"][same]) /
                            np.maximum(1.0, np.abs(r["objective"][same]))))
               if same.any() else None)
    mixed = {"solves_per_s": round(conv_m_all / wall_m, 3),
             "wall_s": round(wall_m, 3), "converged": int(rm["converged"].sum()),
             "fp64_fallbacks": int(rm["fallbacks"]),
             "fp64_inertia_refactorizations": int(rm["inertia_fallbacks"]),
             "max_rel_objective_diff_vs_fp64": obj_dev,
             "max_kkt_error_converged": (float(rm["kkt_error"][rm["converged"]].max())
                                         if rm["converged"].any() else None)}
    seq = []
    for m in B.inst[:sequential_sample]:
        t1 = time.perf_counter()
        one = ipm_driver.solve(ipm_driver.DeviceBackend(
            ipm_driver.CartPoleProblem(m, device), m, device))
        torch.cuda.synchronize()
        seq.append(time.perf_counter() - t1)
    return {"workload": "%d cart-pole instances, N~U{50..400}, one launch per "
                        "IPM phase, FP64" % k,
            "replicas": world, "instances_per_rank": int(B.k),
            "n_total": int(B.n), "nnz_total": int(B.nnz),
            "solves_per_s": round(conv_all / wall, 3),
            "wall_s": round(wall, 3), "setup_s": round(float(r["setup_s"]), 3),
            "converged": int(r["converged"].sum()),
            "unconverged": [int(i) for i in np.nonzero(~r["converged"])[0]],
            "rescued_by_reference_algorithm": int(r["rescued"].sum()),
            "rescued_converged": int((r["rescued"] & r["converged"]).sum()),
            "rescue_note": "instances the batched driver (monotone mu, l1-merit "
                           "line search) leaves unconverged in 200 iterations are "
                           "solved again alone by optimizer.Optimizer (the "
                           "reference's default algorithm) on the GPU core, inside "
                           "the timed region",
            "max_iterations": int(r["iterations"].max()),
            "max_kkt_error": float(r["kkt_error"].max()),
            "mixed": mixed,
            "sequential_single_path_solves_per_s":
                round(len(seq) / float(np.sum(seq)), 3),
            "sequential_sample": "first %d instances, single-problem device "
                                 "path, one after another" % len(seq)}


def ipm_solve_bench(device, solves):
    """Whole interior-point solves of the cart-pole config (N = 100, n = 913)
    on the GPU core: solves/s and latency percentiles over `solves` solves
    after one warm-up solve."""
    import torch
    from amigo_b200 import ipm_driver
    from amigo_b200.problems.cartpole import CartPole
    m = CartPole(N=100, seed=0)
    B = ipm_driver.DeviceBackend(ipm_driver.CartPoleProblem(m, device), m, device)
    r = ipm_driver.solve(B)
    lat = []
    for _ in range(solves):
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = ipm_driver.solve(B)
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t)
    lat = np.array(lat)
    return {"workload": "cart-pole swing-up N=100 (n=913), full IPM solve, FP64",
            "solves_per_s": round(float(len(lat) / lat.sum()), 4),
            "p50_ms": round(1e3 * float(np.percentile(lat, 50)), 2),
            "p99_ms": round(1e3 * float(np.percentile(lat, 99)), 2),
            "iterations": int(r["iterations"]), "objective": r["objective"],
            "kkt_error": r["kkt_error"], "converged": bool(r["converged"]),
            "solves": int(len(lat))}


def ipm_solve_host_baseline():
    """The same driver over the reference's own SparseLDL + IPM vector code
    on the host (oracle/host_backend.py): one solve."""
    from amigo_b200 import ipm_driver
    from amigo_b200.problems.cartpole import CartPole
    from oracle.host_backend import HostBackend
    m = CartPole(N=100, seed=0)
    t = time.perf_counter()
    r = ipm_driver.solve(HostBackend(m))
    dt = time.perf_counter() - t
    return {"solves_per_s": round(1.0 / dt, 4), "iterations": int(r["iterations"]),
            "objective": r["objective"], "kkt_error": r["kkt_error"],
            "kind": "port", "cores": 1,
            "sample": "1 cart-pole N=100 solve with this repository's IPM driver "
                      "(ipm_driver.solve) over a host numeric core: the "
                      "reference's SparseLDL and interior_point_backend.h "
                      "(oracle/_ref) with the numpy restatement of the model's "
                      "derivatives; not the reference's own Optimizer loop"}


def roofline(core, fac_ms):
    """The factorization as one unit (its kernels: per-level small fronts,
    large-front set-up, extend-add, panel and trailing update; the panel
    kernel is the largest share).  Algorithmic bytes of one factorization:
    8 (c(c+1)/2 child-contribution read + f p factor write + c(c+1)/2
    contribution write) per front + 12 nnz(A), over its CUDA-event time."""
    ldl = core.ldl
    h = ldl._h
    npiv, ndel = ldl.node_pivots()
    sym = ldl.symbolic()
    ns = np.diff(sym["node_ptr"])
    nc = np.diff(sym["contrib_ptr"])
    # front sizes: pivots + delayed out + contribution rows; delayed in are
    # the children's delayed out
    kids_ptr, kids = sym["children_ptr"], sym["children"]
    ndin = np.zeros(len(ns))
    for k in range(len(ns)):
        ndin[k] = ndel[kids[kids_ptr[k]:kids_ptr[k + 1]]].sum()
    f = ns + ndin + nc
    p = npiv.astype(float)
    c = f - p
    bytes_ = (8 * (c * (c + 1) / 2 + f * p + c * (c + 1) / 2)).sum() + 12 * core.m.nnz
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_ / (fac_ms * 1e-3) / 1e9
    del h
    return {"kernel": "multifrontal factorization (k_factor_level_rl, k_big_panel, "
                      "k_big_update, k_big_extend, ...; one factorization)",
            "bound": "hbm", "achieved": round(achieved, 2),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 5),
            "traffic": None,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "algorithmic_bytes_per_launch_set": float(bytes_)}


def run_e2e(core, args, device):
    import torch
    m = core.m
    # KKT values and rhs in pinned host memory, copied in every step
    core.fem.hessian(core.vars.x, 1.0, core.K.vals)
    core.K.add_diagonal(core.diag)
    hvals = core.K.vals.cpu().pin_memory()
    hrhs = core.res.cpu().pin_memory()
    hx = torch.empty_like(hrhs).pin_memory()
    flops = core.ldl.stats()["flops"]
    steps = max(3, args.steps // 2)
    stream = torch.cuda.current_stream()
    for _ in range(2):
        core.K.vals.copy_(hvals, non_blocking=True)
        core.ldl.factor()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        core.K.vals.copy_(hvals, non_blocking=True)
        core.ldl.factor()
        core.ldl.get_inertia()
        core.px.copy_(hrhs, non_blocking=True)
        core.ldl.solve_device(core.px)
        hx.copy_(core.px, non_blocking=True)
        torch.cuda.current_stream().synchronize()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    return {"value": round(flops / (ms * 1e-3) / 1e12, 6), "unit": "TFLOP/s",
            "ms_per_step": round(ms, 4),
            "h2d_bytes_per_step": int(8 * (m.nnz + m.n)),
            "d2h_bytes_per_step": int(8 * m.n),
            "work": "per step: KKT values and right-hand side copied in from pinned "
                    "host memory, SparseLDL factor (inertia read back) and one solve, "
                    "solution copied out; `value` times the whole IPM-iteration core "
                    "(element kernels, factor, two solves, refinement, IPM vectors) "
                    "on device-resident data"}


def solve_graph_bench(core, reps=20):
    """Repeated solves on the resident factorization (as refinement steps
    and multi-right-hand-side sensitivities make them): one launch per level
    and sweep against one replay of the captured graph (linalg.SolveGraph),
    CUDA-event time per solve, and whether the replay gave the eager bits."""
    import torch
    from amigo_b200 import linalg
    stream = torch.cuda.current_stream()
    b = core.res.clone()
    x = torch.empty_like(b)
    g = linalg.SolveGraph(core.ldl, x)
    x.copy_(b)
    g()                      # capture
    ref = b.clone()
    core.ldl.solve_device(ref)
    same = bool(torch.equal(x, ref))
    t = {}
    for name, fn in (("eager", lambda: core.ldl.solve_device(x)), ("graph", g)):
        for _ in range(3):
            x.copy_(b)
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        tot = 0.0
        for _ in range(reps):
            x.copy_(b)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        t[name] = round(tot / reps, 4)
    return {"eager_ms_per_solve": t["eager"], "graph_ms_per_solve": t["graph"],
            "replay_bits_equal_eager": same, "captures": g.captures,
            "note": "one solve of the 2D KKT on its resident factorization, "
                    "host-synchronised per solve"}


# ---------------------------------------------------------- reference arm
def kkt_values_host(nx, ny):
    """The same KKT matrix on the host (reference-arm input), from the
    numpy restatement of the model at the same initial point and the same
    barrier diagonal as the GPU step's first factorization."""
    from amigo_b200.problems.simp2d import Simp2D
    from oracle import simp2d_oracle as O
    m = Simp2D(nx, ny)
    x = m.initial_point()
    vals = O.hessian_values(m, x)
    lb, ub = m.lower.copy(), m.upper.copy()
    prim = ~m.mult
    for arr, sgn in ((lb, -1.0), (ub, 1.0)):
        fin = np.isfinite(arr) & prim
        arr[fin] += sgn * np.minimum(1e-4, 1e-8 * np.maximum(1.0, np.abs(arr[fin])))
    d = np.zeros(m.n)
    fl = np.isfinite(lb) & prim
    fu = np.isfinite(ub) & prim
    d[fl] += 1.0 / (x[fl] - lb[fl]).clip(1e-2)
    d[fu] += 1.0 / (ub[fu] - x[fu]).clip(1e-2)
    d[prim] += 1e-8
    vals[m.diag_pos] += d
    vals[m.fixed_diag_pos] = 1.0
    return m, vals


def run_reference_timed(nx, ny, max_seconds, warmup=1, steps=None):
    """The reference's own SparseLDL (oracle/_ref: include/sparse_ldl.h built
    from the reference sources) on this host's cores: factor + solve."""
    from oracle import ref
    m, vals = kkt_values_host(nx, ny)
    cores = os.cpu_count() or 1
    ref.set_blas_threads(1)
    R = ref.RefSparseLDL(m.n, m.rowp, m.cols, order="AMD")
    b = np.ones(m.n)
    for _ in range(warmup):
        R.factor(vals)
        R.solve(b)
    times = []
    t_end = time.time() + max_seconds
    while (steps is None and time.time() < t_end) or (steps is not None and len(times) < steps):
        t = time.time()
        R.factor(vals)
        R.solve(b)
        times.append(time.time() - t)
        if steps is None and len(times) >= 20:
            break
    npiv, ndel = R.node_pivots()
    return m, np.array(times), R, cores


def factor_flops_from_ref(R):
    sym = R.symbolic()
    npiv, ndel = R.node_pivots()
    ns = np.diff(sym["node_ptr"]).astype(float)
    nc = np.diff(sym["contrib_ptr"]).astype(float)
    kp, kids = sym["children_ptr"], sym["children"]
    ndin = np.array([ndel[kids[kp[k]:kp[k + 1]]].sum() for k in range(len(ns))])
    f = ns + ndin + nc
    p = npiv.astype(float)
    c = f - p
    return float((p ** 3 / 3 + p * p * c + p * c * c).sum())


def threads_env():
    """Thread settings of this process (the reference arm's OpenMP tree tasks
    use every core; its BLAS calls are pinned to one thread)."""
    return {"nproc": os.cpu_count(),
            "OMP_NUM_THREADS": os.environ.get("OMP_NUM_THREADS"),
            "OPENBLAS_NUM_THREADS": os.environ.get("OPENBLAS_NUM_THREADS"),
            "reference_blas_threads": 1,
            "reference_openmp": "-fopenmp -DAMIGO_USE_OPENMP"}


def cpu_baseline(nx=128, ny=64):
    m, times, R, cores = run_reference_timed(nx, ny, max_seconds=12.0)
    flops = factor_flops_from_ref(R)
    med = float(np.median(times))
    npiv, _ = R.node_pivots()
    return {"value": round(flops / med / 1e12, 6), "unit": "TFLOP/s",
            "cores": cores, "kind": "reference",
            "inertia": [int(v) for v in R.inertia()], "_npiv": npiv,
            "sample": "%d factor+solve runs of the 2D SIMP 128x64 KKT with the "
                      "reference SparseLDL (AMD, OpenMP tree tasks, 1 BLAS "
                      "thread), median %.3f s" % (len(times), med)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    m, times, R, cores = run_reference_timed(args.nx, args.ny, max_seconds=120.0,
                                             warmup=max(1, min(args.warmup, 2)),
                                             steps=min(args.steps, 10))
    flops = factor_flops_from_ref(R)
    tot = float(np.sum(times))
    value = flops * len(times) / tot / 1e12
    return {
        "metric": METRIC, "impl": "reference", "value": round(value, 6),
        "unit": "TFLOP/s", "n_gpus": world, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": round(1e3 * tot / len(times), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: 2D SIMP KKT at the seeded initial point",
        "config": dict(config(args, 1), n=m.n, nnz=m.nnz),
        "inertia": [int(v) for v in R.inertia()],
        "threads": threads_env(),
        "cpu_baseline": {"value": round(value, 6), "unit": "TFLOP/s",
                         "cores": cores, "kind": "reference",
                         "sample": "reference SparseLDL factor+solve of the full "
                                   "KKT, %d steps" % len(times)},
        "e2e": {"value": round(value, 6), "unit": "TFLOP/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch_under_torchrun(args)
    if world != args.gpus:
        raise SystemExit("bench.py: --gpus %d but WORLD_SIZE=%d" % (args.gpus, world))
    if world > 1:
        import datetime

        import torch
        backend = "nccl" if args.impl == "ours" else "gloo"
        torch.distributed.init_process_group(
            backend, timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world)
        else:
            out = run_ours(args, rank, world, local)
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                from oracle import ref
                if ref.available():
                    cb = cpu_baseline(args.nx, args.ny)
                    rnp = cb.pop("_npiv")
                    out["cpu_baseline"] = cb
                    # parity of the headline KKT: the same matrix factored by
                    # the reference's SparseLDL on the host
                    out["reference_inertia"] = cb["inertia"]
                    out["inertia_equals_reference"] = out["inertia"] == cb["inertia"]
                    if len(rnp) == len(out["_npiv"]):
                        out["pivot_counts_equal_frac"] = round(
                            float(np.mean(rnp == out["_npiv"])), 4)
                    if "ipm_solve" in out:
                        out["ipm_solve"]["host_core_same_driver"] = ipm_solve_host_baseline()
        if rank == 0 and out is not None:
            out.pop("_npiv", None)
            print(json.dumps(out))
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
