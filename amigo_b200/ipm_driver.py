"""A primal-dual interior-point loop over the device numeric core.

amigo's own driver (amigo/algorithm/ipm_driver.py:109-483) is Python that
calls its numeric core; this module is a compact driver of the same shape
for running whole solves on the GPU: residual and KKT error, monotone
barrier update (the reference's "monotone" strategy: reduce mu when
E_mu <= kappa_eps mu, mu <- max(mu_min, min(kappa_mu mu, mu^theta_mu))),
inertia-corrected factorization (Algorithm IC of
amigo/algorithm/inertia_correction.py: increase delta_w until the inertia is
(n_primal, n_constraints), delta_c on the multipliers when the matrix is
singular), Newton direction with 8-block iterative refinement, bound-dual
back-substitution, fraction-to-boundary step, a backtracking line search on
an l1 merit function, and the bound-multiplier reset.  It is not a copy of
amigo's filter line search, watchdog or restoration phase.

The numeric work goes through a backend object; `DeviceBackend` is the
product path (libamigo_b200.so through torch device buffers).  The same
driver runs over a host backend made of the reference's own SparseLDL and
IPM vector functions (oracle/host_backend.py) to compare iteration counts
and optima.
"""
import math
import time

import numpy as np
import torch

from .ipm import InteriorPointOptimizer
from .linalg import OrderingType
from .solver import B200Solver


DEFAULTS = dict(tol=1e-8, max_iter=200, mu0=0.1, mu_min=1e-11,
                kappa_eps=10.0, kappa_mu=0.2, theta_mu=1.5, tau_min=0.99,
                kappa_sigma=1e10, dw_first=1e-4, dw_min=1e-20, dw_max=1e40,
                kw_plus_first=100.0, kw_plus=8.0, kw_minus=1.0 / 3.0,
                dc=1e-8, kappa_c=0.25, armijo=1e-4, max_ls=40,
                refine_steps=1)


def _pw(m, e):
    """m ** e as the device decision kernels evaluate it (csrc/batch_ctrl.cu):
    m * sqrt(m) for 1.5 and sqrt(sqrt(m)) for 0.25, correctly rounded
    square roots on both sides, so host and device decisions agree."""
    if e == 1.5:
        return m * math.sqrt(m)
    if e == 0.25:
        return math.sqrt(math.sqrt(m))
    if e == 1.0:
        return m
    return m ** e


def solve(backend, options=None, verbose=False):
    """Run the interior-point loop; returns a dict with converged,
    iterations, objective, kkt_error, time_s, inertia_corrections."""
    o = dict(DEFAULTS)
    o.update(options or {})
    B = backend
    t0 = time.perf_counter()
    st = B.initial_state()
    mu = o["mu0"]
    dw_last = 0.0
    nu = 1.0
    n_ic = 0
    result = dict(converged=False)
    for it in range(o["max_iter"]):
        g = B.gradient(st)
        d, p, c = B.kkt_error(0.0, st, g)
        E0 = max(d, p, c)
        if verbose:
            print("it %3d  mu %.2e  E0 %.3e  obj %.8e" % (it, mu, E0, B.objective(st)))
        if E0 <= o["tol"]:
            result.update(converged=True, iterations=it)
            break
        # monotone barrier update
        while True:
            Emu = max(B.kkt_error(mu, st, g))
            if Emu <= o["kappa_eps"] * mu and mu > o["mu_min"]:
                mu = max(o["mu_min"], min(o["kappa_mu"] * mu, _pw(mu, o["theta_mu"])))
                continue
            break
        # inertia-corrected factorization
        diag = B.diagonal(st)
        want = (B.np, B.nc)

        def factorize(force_fp64):
            dw, dc, n = 0.0, 0.0, 0
            for attempt in range(41):
                inertia = (B.factor(st, diag, dw, dc, force_fp64=True) if force_fp64
                           else B.factor(st, diag, dw, dc))
                if inertia == want:
                    break
                n += 1
                if inertia[0] + inertia[1] < B.n and dc == 0.0:
                    dc = o["dc"] * _pw(mu, o["kappa_c"])
                if dw == 0.0:
                    dw = o["dw_first"] if dw_last == 0.0 else max(o["dw_min"],
                                                                  o["kw_minus"] * dw_last)
                else:
                    dw *= o["kw_plus_first"] if dw_last == 0.0 else o["kw_plus"]
                if dw > o["dw_max"]:
                    break
            return dw, n

        dw, n = factorize(False)
        n_ic += n
        # Newton direction
        res = B.residual(mu, st, g)
        px = B.solve(res)
        if o["refine_steps"] and not B.refine(mu, st, g, res, px, o["refine_steps"]):
            # the FP32 factor's inertia was accepted but the FP64 factor of
            # the same matrix has another one: correct the inertia in FP64
            dw, n = factorize(True)
            n_ic += n
            res = B.residual(mu, st, g)
            px = B.solve(res)
            B.refine(mu, st, g, res, px, o["refine_steps"])
        if dw > 0.0:
            dw_last = dw
        upd = B.update(mu, st, px)
        tau = max(o["tau_min"], 1.0 - mu)
        ax, az = B.max_step(tau, st, upd)
        # l1-merit backtracking line search
        nu = max(nu, 1.1 * B.max_abs_mult(st, px))
        gf = B.objective_gradient(st)
        theta0 = B.cviol(st, g)
        phi0 = B.objective(st) + B.barrier_log_sum(mu, st) + nu * theta0
        dphi = B.dphi(mu, st, gf, px) - nu * theta0
        alpha = ax
        trial = None
        for ls in range(o["max_ls"]):
            trial = B.apply_step(alpha, az, st, upd)
            gt = B.gradient(trial)
            phi = B.objective(trial) + B.barrier_log_sum(mu, trial) + nu * B.cviol(trial, gt)
            if phi <= phi0 + o["armijo"] * alpha * dphi or not math.isfinite(dphi):
                break
            alpha *= 0.5
        st = trial
        B.reset_bound_multipliers(mu, o["kappa_sigma"], st)
    else:
        result.update(iterations=o["max_iter"])
    g = B.gradient(st)
    result.update(objective=B.objective(st), kkt_error=max(B.kkt_error(0.0, st, g)),
                  time_s=time.perf_counter() - t0, inertia_corrections=n_ic,
                  x=B.solution(st))
    return result


def solve_batch(model, device="cuda", options=None, verbose=False,
                precision="fp64", rescue=True, rescue_workers=4):
    """`solve` for every instance of a batch (problems.cartpole.CartPoleBatch)
    at once, on batch_engine.BatchEngine: each phase is one launch over all
    instances (the KKT matrices are factored together by the block-diagonal
    multifrontal LDL^T), while the barrier parameter, inertia correction,
    refinement stopping rule, step lengths and line search are kept per
    instance, so each instance takes the decisions it would take alone.  An
    instance that has converged takes no further steps.  Returns a dict of
    per-instance arrays: converged, iterations, objective, kkt_error,
    inertia_corrections, plus time_s (all of it), setup_s (symbolic
    analysis, uploads), fallbacks (FP64 refactorizations of the
    mixed-precision form after a stalled refinement), inertia_fallbacks
    (FP64 refactorizations on an FP32 inertia mismatch) and x (host,
    concatenated).  precision "fp32" factors with FP32 fronts and refines
    every direction against the FP64 KKT.  With `rescue`, an instance the
    batched driver leaves unconverged is solved again, alone, by
    optimizer.Optimizer (amigo's default algorithm: heuristic barrier,
    filter line search, restoration) on the same GPU core; `rescued` marks
    them (their time is part of time_s).  The re-solves run on
    `rescue_workers` host threads, each with its own CUDA stream (every
    re-solve is independent, so the results are those of the re-solves one
    after another)."""
    from .batch_engine import BatchEngine
    dev = torch.device(device)
    t0 = time.perf_counter()
    eng = BatchEngine(dev, options, precision)
    eng.admit(enumerate(model.inst))
    eng._build()
    torch.cuda.synchronize(dev)
    t_setup = time.perf_counter() - t0
    results = {}
    while len(results) < model.k:
        # compact the layout once half of it has retired, so the last
        # instances' iterations factor only the live ones
        for r in eng.step(rebuild=eng.live() > 0 and eng.dead_fraction() >= 0.5):
            results[r["id"]] = r
        if verbose:
            print("live %d" % (model.k - len(results)))
    R = [results[k] for k in range(model.k)]
    rescued = np.zeros(model.k, bool)
    if rescue:
        todo = [k for k, r in enumerate(R) if not r["converged"]]
        for k, r in zip(todo, _solve_reference_algorithm_many(
                [model.inst[k] for k in todo], dev, rescue_workers)):
            R[k] = r
            rescued[k] = True
    col = lambda key, dt: np.array([r[key] for r in R], dtype=dt)
    return dict(converged=col("converged", bool), iterations=col("iterations", np.int64),
                objective=col("objective", float), kkt_error=col("kkt_error", float),
                inertia_corrections=col("inertia_corrections", np.int64),
                time_s=time.perf_counter() - t0, setup_s=t_setup, rescued=rescued,
                fallbacks=eng.fallbacks, inertia_fallbacks=eng.inertia_fallbacks,
                x=np.concatenate([r["x"] for r in R]))


def _solve_reference_algorithm_many(models, dev, workers):
    """_solve_reference_algorithm for each model, on up to `workers` host
    threads with one CUDA stream per thread (the library's calls take the
    thread's current stream; its reductions keep scratch per stream)."""
    if not models:
        return []
    if workers <= 1 or len(models) == 1:
        return [_solve_reference_algorithm(m, dev) for m in models]
    import threading
    from concurrent.futures import ThreadPoolExecutor
    local = threading.local()

    def run(m):
        s = getattr(local, "stream", None)
        if s is None:
            s = local.stream = torch.cuda.Stream(device=dev)
        with torch.cuda.stream(s):
            r = _solve_reference_algorithm(m, dev)
            s.synchronize()
        return r

    torch.cuda.synchronize(dev)
    with ThreadPoolExecutor(max_workers=min(workers, len(models))) as ex:
        return list(ex.map(run, models))


def _solve_reference_algorithm(m, dev):
    """One cart-pole instance by optimizer.Optimizer on the GPU core."""
    from .optimizer import Optimizer
    P = CartPoleProblem(m, dev)
    x = torch.from_numpy(np.asarray(m.x0, dtype=np.float64)).to(dev)
    opt = Optimizer(P, x, np.asarray(m.lower, np.float64), np.asarray(m.upper, np.float64),
                    B200Solver(P), device=dev)
    r = opt.optimize()
    xf = opt.vars.get_solution()
    last = r["iterations"][-1]
    return dict(converged=bool(r["converged"]), iterations=len(r["iterations"]) - 1,
                objective=P.objective(xf), kkt_error=float(last["nlp_error"]),
                inertia_corrections=int(sum(1 for it in r["iterations"]
                                            if it.get("inertia_delta", 0.0) > 0.0)),
                x=xf.cpu().numpy())


class CartPoleProblem:
    """Device KKT problem for a model whose device_model() gives gradient,
    hessian and objective(x, out) kernels: the cart-pole model
    (problems/cartpole.py) or a generated component model
    (codegen.GeneratedModel)."""

    def __init__(self, model, device="cuda"):
        from .linalg import CSRMat
        self.model = model
        self.device = torch.device(device)
        self.dm = model.device_model(self.device)
        self._csr = CSRMat
        self._obj = torch.zeros(1, dtype=torch.float64, device=self.device)

    def get_multiplier_indicator(self):
        return self.model.mult

    def create_matrix(self):
        m = self.model
        return self._csr(m.n, m.n, m.rowp, m.cols, device=self.device)

    def hessian(self, alpha, x, hess):
        self.dm.hessian(x, alpha, hess.vals)

    def gradient(self, alpha, x, g):
        self.dm.gradient(x, alpha, g)

    def add_diagonal(self, diag, hess):
        hess.add_diagonal(diag)

    def objective(self, x):
        self.dm.objective(x, self._obj)
        return float(self._obj.item())

    def create_vector(self):
        return torch.zeros(self.model.n, dtype=torch.float64, device=self.device)

    def lagrangian(self, alpha, x):
        """alpha f(x) + lambda^T c(x) (include/optimization_problem.h
        lagrangian): the multiplier rows of the gradient are c(x)."""
        return alpha * self.objective(x) + _multiplier_term(self, x)

    def update(self, x):
        pass


def _multiplier_term(p, x):
    if not hasattr(p, "_g_tmp"):
        p._g_tmp = torch.zeros(p.model.n, dtype=torch.float64, device=p.device)
        p._mult_idx = torch.from_numpy(
            np.nonzero(np.asarray(p.model.mult, bool))[0]).to(p.device)
    p.gradient(1.0, x, p._g_tmp)
    i = p._mult_idx
    return float(torch.dot(x[i], p._g_tmp[i]).item())


GeneratedProblem = CartPoleProblem


class SimpProblem:
    """Device KKT problem for the SIMP compliance models (problems/simp2d.py,
    problems/simp3d.py); the objective is the compliance f^T u."""

    def __init__(self, model, device="cuda"):
        from .linalg import CSRMat
        self.model = model
        self.device = torch.device(device)
        self.dm = model.device_model(self.device)
        self._csr = CSRMat
        self._f = torch.from_numpy(np.ascontiguousarray(model.f)).to(self.device)

    def get_multiplier_indicator(self):
        return self.model.mult

    def create_matrix(self):
        m = self.model
        return self._csr(m.n, m.n, m.rowp, m.cols, device=self.device,
                         diag_pos=m.diag_pos)

    def hessian(self, alpha, x, hess):
        self.dm.hessian(x, alpha, hess.vals)

    def gradient(self, alpha, x, g):
        self.dm.gradient(x, alpha, g)

    def add_diagonal(self, diag, hess):
        hess.add_diagonal(diag)

    def objective(self, x):
        return float(torch.dot(self._f, x).item())

    def create_vector(self):
        return torch.zeros(self.model.n, dtype=torch.float64, device=self.device)

    def lagrangian(self, alpha, x):
        """alpha f(x) + lambda^T c(x), as CartPoleProblem.lagrangian."""
        return alpha * self.objective(x) + _multiplier_term(self, x)

    def update(self, x):
        pass


class DeviceBackend:
    """Numeric core on the GPU: component kernels, multifrontal LDL^T,
    IPM vector kernels.

    precision "fp32" is the mixed-precision form: the KKT is factored with
    FP32 fronts (tensor-core Schur updates on large fronts), every Newton
    direction gets at least `mixed_refine_steps` steps of the 8-block
    iterative refinement against the FP64 KKT, and an iteration whose
    refinement stalls above 1e-10 is refactored in FP64 and solved again
    (counted in `fallbacks`)."""

    mixed_refine_steps = 4

    def __init__(self, problem, model, device="cuda", precision="fp64"):
        self.P = problem
        self.m = model
        self.device = torch.device(device)
        self.precision = precision
        self.fallbacks = 0          # stalled FP32 refinements redone in FP64
        self.inertia_fallbacks = 0  # FP32 inertia mismatches refactored in FP64
        self.fp64_now = precision != "fp32"
        self.solver = B200Solver(problem, order=OrderingType.AMD,
                                 precision=precision)
        self.opt = InteriorPointOptimizer(model.mult, model.lower, model.upper,
                                          device=self.device)
        self.opt.relax_bounds()
        self.n, self.np, self.nc = model.n, self.opt.np_, self.opt.nc_
        f64 = dict(dtype=torch.float64, device=self.device)
        self.g = torch.zeros(self.n, **f64)
        self.gf = torch.zeros(self.n, **f64)
        self.res = torch.zeros(self.n, **f64)
        self.px = torch.zeros(self.n, **f64)
        self.diag = torch.zeros(self.n, **f64)
        self.dtot = torch.zeros(self.n, **f64)
        self.primal = torch.from_numpy(~model.mult).to(self.device).double()
        self.upd = self.opt.create_opt_vector()
        self.xtmp = torch.zeros(self.n, **f64)
        self._hsave = None
        self._hx = None
        self.mult_idx = self.opt.cidx.long()
        self._lbx = self.opt.lbx.cpu().numpy()
        self._ubx = self.opt.ubx.cpu().numpy()

    def initial_state(self):
        x = torch.from_numpy(np.ascontiguousarray(self.m.x0)).to(self.device)
        v = self.opt.create_opt_vector(x)
        self.opt.initialize_multipliers_and_slacks(0.1, None, v)
        return v

    def _new_state(self):
        return self.opt.create_opt_vector()

    def gradient(self, st):
        out = torch.zeros(self.n, dtype=torch.float64, device=self.device)
        self.P.gradient(1.0, st.x, out)
        return out

    def objective_gradient(self, st):
        self.xtmp.copy_(st.x)
        self.xtmp[self.mult_idx] = 0.0
        self.P.gradient(1.0, self.xtmp, self.gf)
        return self.gf

    def objective(self, st):
        return self.P.objective(st.x)

    def kkt_error(self, mu, st, g):
        return self.opt.compute_kkt_error_mu(mu, st, g)

    def diagonal(self, st):
        self.opt.compute_diagonal(st, self.diag)
        return self.diag

    def factor(self, st, diag, dw, dc, force_fp64=False):
        """Factor K + diag(diag + dw on primals - dc on multipliers); returns
        the inertia.  FP32 fronts are kept only when their inertia is the
        one the inertia correction wants, (n_primal, n_constraints): a
        mismatch may be an FP32 artefact (eigenvalues below FP32
        resolution), so the correction loop decides on the FP64 factor's
        inertia instead."""
        torch.add(diag, self.primal, alpha=dw, out=self.dtot)
        if dc:
            self.dtot.sub_(1.0 - self.primal, alpha=dc)
        self._fx = st.x
        self.fp64_now = self.precision != "fp32" or force_fp64
        if self.precision == "fp32" and force_fp64:
            self.solver.set_precision("fp64")
        self.solver.factor(1.0, st.x, self.dtot)
        inertia = self.solver.get_inertia()
        if self.precision == "fp32" and not force_fp64 and inertia != (self.np, self.nc):
            self.inertia_fallbacks += 1
            self.solver.set_precision("fp64")
            self.solver.factor(1.0, st.x, self.dtot)
            inertia = self.solver.get_inertia()
            self.fp64_now = True
        if self.precision == "fp32":
            self.solver.set_precision("fp32")
        return inertia

    def residual(self, mu, st, g):
        self.opt.compute_residual(mu, st, g, self.res)
        return self.res

    def solve(self, res):
        self.solver.solve(res, self.px)
        return self.px

    def refine(self, mu, st, g, res, px, steps):
        """Iterative refinement of the Newton direction px.  Returns False
        when the FP32 factor's refinement stalled and the FP64
        refactorization of the same matrix has an inertia other than
        (n_primal, n_constraints): the caller then redoes the inertia
        correction on FP64 factors."""
        mixed = self.precision == "fp32" and not self.fp64_now
        if mixed:
            steps = max(steps, self.mixed_refine_steps)
        self.solver.iterative_refinement(mu, self.m.mult, res, st, g,
                                         self._lbx, self._ubx, px, None, None,
                                         max_steps=steps + 1)
        if mixed and self.solver.last_refinement[1] > 1e-10:
            # refinement stalled on the FP32 factor: refactor in FP64
            self.fallbacks += 1
            self.solver.set_precision("fp64")
            self.solver.factor(1.0, self._fx, self.dtot)
            self.fp64_now = True
            self.solver.set_precision("fp32")
            if self.solver.get_inertia() != (self.np, self.nc):
                return False
            self.solver.solve(res, px)
            self.solver.iterative_refinement(mu, self.m.mult, res, st, g,
                                             self._lbx, self._ubx, px, None,
                                             None, max_steps=steps + 1)
        return True

    def update(self, mu, st, px):
        self.opt.compute_update(mu, st, px, self.upd)
        return self.upd

    def max_step(self, tau, st, upd):
        ax, xi, az, zi = self.opt.compute_max_step(tau, st, upd)
        return ax, az

    def apply_step(self, ax, az, st, upd):
        t = self._new_state()
        t.copy(st)
        self.opt.apply_step_update(ax, az, st, upd, t)
        return t

    def max_abs_mult(self, st, px):
        lam = st.x[self.mult_idx] + px[self.mult_idx]
        return float(lam.abs().max().item()) if lam.numel() else 0.0

    def cviol(self, st, g):
        return self.opt.compute_constraint_violation_1norm(st, g)

    def barrier_log_sum(self, mu, st):
        return self.opt.compute_barrier_log_sum(mu, st)

    def dphi(self, mu, st, gf, px):
        return self.opt.compute_barrier_dphi_direct(mu, st, gf, px)

    def reset_bound_multipliers(self, mu, kappa, st):
        self.opt.reset_bound_multipliers(mu, kappa, st)

    def solution(self, st):
        return st.x.cpu().numpy()
