"""Interior-point driver over the InteriorPointOptimizer / LinearSolver /
problem interfaces, making amigo's default algorithmic decisions.

amigo's `Optimizer` (amigo/algorithm/ipm_driver.py:109-483 with the modules
it composes) is host control flow over three interfaces: the backend
(InteriorPointOptimizer), the linear solver and the problem.  This module
takes the same decisions with the same default options -- so that an
amigo user who moves the numeric core to the GPU keeps the iterates,
iteration counts and optima of the reference -- in a driver written for
this package:
  * start point: bound relaxation, interior projection, unit bound duals,
    NLP scaling (objective and constraint rows), least-squares constraint
    multipliers with the |y| <= 1e3 safeguard (iterate_initialization.py,
    multiplier_initialization.py:17-52);
  * barrier: the LOQO-type heuristic mu = gamma * min(2, (1 - r)(1 - xi)
    / xi)^3 * avg_complementarity, floored at min(tol, compl_tol) /
    (kappa_eps + 1) (barrier_strategy/heuristic.py:53-105);
  * Newton direction: Algorithm IC inertia correction with its
    degeneracy tests (inertia_correction.py:31-402), the condensed
    residual, the solve and the solver's 8-block iterative refinement
    (newton_direction.py:95-131);
  * globalisation: fraction to the boundary with tau = max(tau_min,
    1 - mu), the filter line search over (barrier objective, 1-norm
    constraint violation) with second-order corrections and the watchdog
    (filter_line_search.py, filter_acceptance.py), feasibility restoration
    when the line search fails (feasibility_restoration.py), slack
    flooring and the bound-multiplier reset (bound_safeguards.py);
  * termination: the scaled KKT error with the acceptable-point, divergence
    and precision-floor tests (convergence_check.py, optimality_scaling.py).
The constants and tests are the reference's, because the iteration
sequence depends on every one of them.

Vectors are whatever the problem creates: device tensors (amigo_b200's
InteriorPointOptimizer, B200Solver and device problems) or objects with a
get_array() view (a host numeric core).  `_a` returns the array either
way, and the few array operations the driver makes work on numpy arrays
and torch tensors alike.
"""
import math
import time

import numpy as np

try:
    import torch
except ImportError:  # a host core needs no torch
    torch = None

# amigo's options whose default values are the default algorithm that
# this driver restates (amigo/algorithm/default_options.py): they are
# accepted at these values; other values select strategies (adaptive or
# quality-function barrier updates, Armijo-only line search, adaptive
# regularisation settings, ...) that are not restated.
DEFAULT_ALGORITHM_OPTIONS = {
    "adaptive_mu_globalization": "obj-constr-filter", "adaptive_mu_kkterror_red_fact": 0.9999,
    "adaptive_mu_kkterror_red_iters": 4, "adaptive_mu_monotone_init_factor": 0.8,
    "adaptive_mu_safeguard_factor": 0.0, "adaptive_regularization": True,
    "armijo_constant": 1e-4, "barrier_progress_tol": 10.0, "barrier_strategy": "heuristic",
    "check_update_step": False, "continuation_control": None, "debug_cycling": False,
    "equal_primal_dual_step": False, "filter_line_search": True,
    "init_affine_step_multipliers": False, "max_regularization": 0.01,
    "monotone_barrier_fraction": 0.1, "mu_linear_decrease_factor": 0.2,
    "mu_max_fact": 1000.0, "mu_min": 1e-11, "mu_superlinear_decrease_power": 1.5,
    "progress_based_barrier": True, "quality_function_balancing_term": "none",
    "quality_function_centrality": "none", "quality_function_golden_iters": 8,
    "quality_function_norm_scaling": True, "quality_function_predictor_corrector": False,
    "quality_function_section_qf_tol": 0.0, "quality_function_section_sigma_tol": 0.01,
    "quality_function_sigma_max": 100.0, "quality_function_sigma_min": 1e-6,
    "record_components": [], "regularization_eps_x": 1e-8,
    "regularization_eps_x_zero_hessian": 1.0, "regularization_eps_z": 1e-8,
    "regularization_increase_factor": 10.0, "use_armijo_line_search": True,
    "verbose_barrier": False, "zero_hessian_variables": [],
}
# of these, the ones that only change what is printed or recorded
DIAGNOSTIC_OPTIONS = ("debug_cycling", "verbose_barrier", "record_components")

DEFAULT_OPTIONS = dict(
    max_iterations=100, convergence_tolerance=1e-8, dual_inf_tol=1.0,
    constr_viol_tol=1e-4, compl_inf_tol=1e-4, diverging_iterates_tol=1e20,
    fraction_to_boundary=0.99, initial_barrier_param=1.0,
    max_line_search_iterations=40, backtracking_factor=0.5,
    init_least_squares_multipliers=True, heuristic_barrier_gamma=0.1,
    heuristic_barrier_r=0.95, barrier_tol_factor=10.0,
    filter_gamma_theta=1e-5, filter_gamma_phi=1e-8, filter_delta=1.0,
    filter_s_theta=1.1, filter_s_phi=2.3, filter_eta_phi=1e-8, filter_max_soc=4,
    filter_kappa_soc=0.99, filter_restoration_max_iter=20, filter_reset_trigger=5,
    max_filter_resets=5, watchdog_shortened_iter_trigger=10,
    watchdog_trial_iter_max=3, acceptable_tol=1e-6, acceptable_iter=15,
    acceptable_dual_inf_tol=1e10, acceptable_constr_viol_tol=1e-2,
    acceptable_compl_inf_tol=1e-2, adaptive_tau=True, tau_min=0.99,
    max_consecutive_rejections=5, barrier_increase_factor=5.0,
    max_inertia_corrections=40, inertia_tolerance=0,
    nlp_scaling_max_gradient=100.0, second_order_correction=True,
)

CONTINUE, CONVERGED, ACCEPTABLE, DIVERGED, FLOOR = range(5)
_EPS = np.finfo(np.float64).eps


# ---------------------------------------------------------------- arrays
def _a(v):
    """The array behind a vector object (host numpy or device tensor)."""
    if torch is not None and isinstance(v, torch.Tensor):
        return v
    if hasattr(v, "dev"):          # amigo_b200.linalg.Vector
        return v.dev
    if hasattr(v, "arr"):          # host vector
        return v.arr
    return v.get_array()


def _copy(a):
    return a.clone() if (torch is not None and isinstance(a, torch.Tensor)) else a.copy()


def _host(a):
    if torch is not None and isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _sync(v):
    """Host -> device copy for vectors that keep a host mirror."""
    if hasattr(v, "copy_host_to_device") and not hasattr(v, "dev"):
        v.copy_host_to_device()


class _Filter:
    """(phi, theta) filter with the margins added at insertion
    (filter_acceptance.py): phi - gamma_phi theta, (1 - gamma_theta) theta."""

    def __init__(self, gamma_phi, gamma_theta):
        self.gp, self.gt = gamma_phi, gamma_theta
        self.pts = []

    def acceptable(self, phi, theta):
        return not any(phi > p and theta > t for p, t in self.pts)

    def add(self, phi, theta):
        pe, te = phi - self.gp * theta, (1.0 - self.gt) * theta
        self.pts = [(p, t) for p, t in self.pts if not (p >= pe and t >= te)]
        self.pts.append((pe, te))

    def clear(self):
        self.pts = []


class InertiaCorrection:
    """Algorithm IC (Wachter & Biegler 2006): grow delta_w (primal) and
    add delta_c (constraint) regularisation until the factor has inertia
    (n_primal, n_constraints), with the structural-degeneracy tests that
    carry decisions from one iteration to the next."""

    NOT_YET, NOT_DEGEN, DEGEN = 0, 1, 2
    NONE, DC0_DX0, DC1_DX0, DC0_DX1, DC1_DX1 = range(5)

    def __init__(self, mult, mu):
        self.mult = np.asarray(mult, bool)
        self.mu = mu
        self.dx_last = self.dc_last = 0.0
        self.dx = self.dc = 0.0
        self.last_delta_w = self.last_delta_c = 0.0
        self.hess_degen = self.jac_degen = self.NOT_YET
        self.degen_iters = 0
        self.test = self.NONE
        self.pivtol = 1e-6

    def _dcd(self):
        return 1e-8 * self.mu ** 0.25

    def _grow(self):
        prev = self.dx
        if self.dx == 0.0:
            # the reference's decrease factor is the double 1/3 (a product,
            # not a division: the two differ in the last bit)
            self.dx = 1e-4 if self.dx_last == 0.0 else max(1e-20, self.dx_last * (1.0 / 3))
        elif self.dx_last == 0.0 or 1e5 * self.dx_last < self.dx:
            self.dx *= 100.0
        else:
            self.dx *= 8.0
        if self.dx > 1e20:
            self.dx = prev
            self.dx_last = 0.0
            return False
        return True

    def _conclude(self):
        t = self.test
        if t == self.DC0_DX0:
            if self.hess_degen == self.NOT_YET:
                self.hess_degen = self.NOT_DEGEN
            if self.jac_degen == self.NOT_YET:
                self.jac_degen = self.NOT_DEGEN
        elif t == self.DC1_DX0:
            if self.hess_degen == self.NOT_YET:
                self.hess_degen = self.NOT_DEGEN
            if self.jac_degen == self.NOT_YET:
                self.degen_iters += 1
                if self.degen_iters >= 3:
                    self.jac_degen = self.DEGEN
        elif t == self.DC0_DX1:
            if self.jac_degen == self.NOT_YET:
                self.jac_degen = self.NOT_DEGEN
            if self.hess_degen == self.NOT_YET:
                self.degen_iters += 1
                if self.degen_iters >= 3:
                    self.hess_degen = self.DEGEN
        elif t == self.DC1_DX1:
            self.degen_iters += 1
            if self.degen_iters >= 3:
                self.hess_degen = self.jac_degen = self.DEGEN
        self.test = self.NONE

    def _new_system(self):
        self._conclude()
        if self.dx > 0.0:
            self.dx_last = self.dx
        if self.dc > 0.0:
            self.dc_last = self.dc
        undecided = self.NOT_YET in (self.hess_degen, self.jac_degen)
        self.test = self.DC0_DX0 if undecided else self.NONE
        self.dc = self._dcd() if self.jac_degen == self.DEGEN else 0.0
        self.dx = 0.0
        if self.hess_degen == self.DEGEN:
            self._grow()

    def _wrong_inertia(self):
        self._conclude()
        if self._grow():
            return True
        if self.dc == 0.0:
            self.dc = self._dcd()
            self.dx = 0.0
            if self.hess_degen == self.DEGEN:
                self.hess_degen = self.NOT_YET
            self.test = self.NONE
            return self._grow()
        return False

    def _singular(self):
        if self.NOT_YET in (self.hess_degen, self.jac_degen):
            t = self.test
            if t == self.DC0_DX0:
                if self.jac_degen == self.NOT_YET:
                    self.dc = self._dcd()
                    self.test = self.DC1_DX0
                else:
                    if not self._grow():
                        return False
                    self.test = self.DC0_DX1
            elif t == self.DC1_DX0:
                self.dc = 0.0
                if not self._grow():
                    return False
                self.test = self.DC0_DX1
            elif t == self.DC0_DX1:
                self.dc = self._dcd()
                if not self._grow():
                    return False
                self.test = self.DC1_DX1
            elif t == self.DC1_DX1:
                if not self._grow():
                    return False
        elif self.dc > 0.0:
            if not self._grow():
                return False
        else:
            self.dc = self._dcd()
        return True

    def factorize(self, solver, x, diag, obj_scale, scaling_fn, max_corrections=40,
                  tolerance=0):
        """Assemble H at x, then factor H + diag(diag + eps + dx on primals
        - dc on constraints) until the inertia is right.  Returns True on
        success, False when the corrections run out."""
        solver.assemble_hessian(obj_scale, x)
        if scaling_fn is not None:
            scaling_fn(solver.hess)
        prim = ~self.mult
        npr, nd = int(prim.sum()), int(self.mult.sum())
        d = _a(diag)
        pm = self._mask(prim, d)
        mm = self._mask(self.mult, d)
        d[pm] += 1e-12
        _sync(diag)
        base = _copy(d)
        self._new_system()
        quality_raised = False
        for attempt in range(max_corrections + 1):
            d[...] = base
            if self.dx > 0:
                d[pm] += self.dx
            if self.dc > 0:
                d[mm] -= self.dc
            _sync(diag)
            singular = False
            try:
                if attempt == 0:
                    solver.add_diagonal_and_factor(diag)
                else:
                    solver.factor(obj_scale, x, diag, post_hessian=scaling_fn)
                npos, nneg = solver.get_inertia()
            except Exception:
                npos = nneg = 0
                singular = True
            if not singular and abs(npos - npr) <= tolerance and \
                    abs(nneg - nd) <= tolerance and npos + nneg >= npr + nd - tolerance:
                self.last_delta_w, self.last_delta_c = self.dx, self.dc
                return True
            if singular and nd > 0:
                if not self._singular():
                    break
            elif not singular and nneg < nd:
                # too few negative eigenvalues: raise the pivot quality
                # once, else treat the matrix as singular
                if not quality_raised and self.pivtol < 0.1:
                    self.pivtol = min(0.1, self.pivtol ** 0.5)
                    quality_raised = True
                elif not self._singular():
                    break
            elif not self._wrong_inertia():
                break
        self.last_delta_w, self.last_delta_c = self.dx, self.dc
        return False

    _masks = {}

    @classmethod
    def _mask(cls, m, like):
        """The boolean mask m as an index for `like` (its device copy for a
        tensor, cached; the cache holds m itself, so its id stays unique)."""
        if torch is not None and isinstance(like, torch.Tensor):
            key = (id(m), str(like.device))
            hit = cls._masks.get(key)
            if hit is None or hit[0] is not m:
                hit = (m, torch.from_numpy(np.ascontiguousarray(m)).to(like.device))
                cls._masks[key] = hit
            return hit[1]
        return m


class _Watchdog:
    def __init__(self, ipo, trigger, max_trials):
        self.on = False
        self.shortened = 0
        self.trials = 0
        self.trigger, self.max_trials = trigger, max_trials
        self.upd = ipo.create_opt_vector()
        self.x = self.px = None
        self.alpha = self.theta = self.barr = self.dphi = 0.0

    def reset(self):
        self.on = False
        self.shortened = self.trials = 0
        self.x = self.px = None


class Optimizer:
    """Optimizer(problem, x, lower, upper, solver, backend_class).optimize()

    problem: gradient(alpha, x, g), hessian(alpha, x, H), add_diagonal,
    create_vector, create_matrix, lagrangian(alpha, x),
    get_multiplier_indicator; solver: a LinearSolver with inertia and
    iterative_refinement (B200Solver); backend_class: the
    InteriorPointOptimizer class, constructed as (problem, lower, upper)."""

    def __init__(self, problem, x, lower, upper, solver, backend_class=None,
                 **backend_kw):
        if backend_class is None:
            from .ipm import InteriorPointOptimizer as backend_class
        self.problem = problem
        self.solver = solver
        self.ipo = backend_class(problem, lower, upper, **backend_kw)
        self.mult = np.asarray(problem.get_multiplier_indicator(), bool)
        self.x0 = x
        self.vars = self.ipo.create_opt_vector(x)
        self.update = self.ipo.create_opt_vector()
        self.temp = self.ipo.create_opt_vector()
        self.grad, self.res, self.diag, self.px, self.ir_corr = (
            problem.create_vector() for _ in range(5))
        self.mu = 1.0
        self.obj_scale = 1.0
        self.scale_fn = None

    # -- evaluations ----------------------------------------------------------
    def _sol(self, v=None):
        return (v or self.vars).get_solution()

    def _gradient(self, x):
        if hasattr(self.problem, "update"):
            self.problem.update(x)
        self.problem.gradient(self.obj_scale, x, self.grad)
        self.ipo.apply_gradient_scaling(self.grad)

    def _theta(self, v=None):
        return self.ipo.compute_constraint_violation_1norm(v or self.vars, self.grad)

    def _barrier_objective(self, v):
        """phi_mu = f(x) - mu sum log(gaps), f from L(x, lam = 0)."""
        xv = v.get_solution()
        xa = _a(xv)
        m = InertiaCorrection._mask(self.mult, xa)
        lam = _copy(xa[m])
        xa[m] = 0.0
        _sync(xv)
        f = float(self.problem.lagrangian(self.obj_scale, xv))
        xa[m] = lam
        _sync(xv)
        return f + self.ipo.compute_barrier_log_sum(self.mu, v)

    def _scaling(self):
        """(s_d, s_c) of the scaled optimality error (s_max = 100)."""
        zl = np.abs(np.asarray(self.vars.get_zl(), dtype=np.float64)).sum()
        zu = np.abs(np.asarray(self.vars.get_zu(), dtype=np.float64)).sum()
        z = float(zl + zu)
        nb = self._nbounds
        xa = _a(self._sol())
        y = float(np.abs(_host(xa[InertiaCorrection._mask(self.mult, xa)])).sum())
        nc = int(self.mult.sum())
        s_c = 1.0 if nb == 0 else max(100.0, z / nb) / 100.0
        s_d = 1.0 if nc + nb == 0 else max(100.0, (y + z) / (nc + nb)) / 100.0
        return s_d, s_c

    def _kkt_error(self):
        d, p, c = self.ipo.compute_kkt_error_mu(0.0, self.vars, self.grad)
        s_d, s_c = self._scaling()
        return max(d / s_d, p, c / s_c), d, p, c

    # -- start point ------------------------------------------------------------
    def _initialize(self, o):
        ipo = self.ipo
        x = self._sol()
        ipo.relax_bounds(1e-8, o["constr_viol_tol"])
        ipo.set_multipliers_value(0.0, x)
        ipo.initialize_multipliers_and_slacks(self.mu, self.grad, self.vars)
        if ipo.has_slacks():
            self._gradient(x)
            ipo.initialize_slacks(self.grad, self.vars)
            _sync(x)
            ipo.initialize_multipliers_and_slacks(self.mu, self.grad, self.vars)
        self._gradient(x)
        if o["nlp_scaling_max_gradient"] > 0:
            ipo.compute_nlp_scaling(x, self.grad, max_gradient=o["nlp_scaling_max_gradient"])
            self.obj_scale = ipo.get_obj_scale()
            if ipo.has_scaling():
                self.scale_fn = ipo.apply_hessian_scaling
                self._gradient(x)
        if o["init_least_squares_multipliers"]:
            self._least_squares_multipliers()
        self._gradient(x)

    def _least_squares_multipliers(self, lam_max=1e3):
        """y minimising the dual infeasibility: solve [I A^T; A 0] [w; y] =
        [-(grad_f - zl + zu); 0]; y = 0 if |y|_inf > lam_max."""
        ipo, x = self.ipo, self._sol()
        ipo.compute_dual_residual_vector(self.vars, self.grad, self.res)
        r = _a(self.res)
        r *= -1.0
        _sync(self.res)
        d = _a(self.diag)
        d[...] = 0.0
        ipo.set_design_vars_value(1.0, self.diag)
        _sync(self.diag)
        self.solver.factor(0.0, x, self.diag, post_hessian=self.scale_fn)
        self.solver.solve(self.res, self.px)
        pa = _a(self.px)
        lam = np.abs(_host(pa[InertiaCorrection._mask(self.mult, pa)]))
        if lam.size and float(lam.max()) > lam_max:
            ipo.set_multipliers_value(0.0, x)
            return
        ipo.copy_multipliers(x, self.px)

    # -- Newton direction ---------------------------------------------------------
    def _direction(self, x, diag_base, ic, o):
        d = _a(self.diag)
        d[...] = diag_base
        _sync(self.diag)
        ok = ic.factorize(self.solver, x, self.diag, self.obj_scale, self.scale_fn,
                          o["max_inertia_corrections"], o["inertia_tolerance"])
        if not ok:
            return False
        self._solve(self.mu)
        return True

    def _solve(self, mu):
        ipo = self.ipo
        ipo.compute_residual(mu, self.vars, self.grad, self.res)
        rhs = _copy(_a(self.res))
        self.solver.solve(self.res, self.px)
        lbx = np.asarray(ipo.get_lbx_relaxed(), dtype=np.float64)
        ubx = np.asarray(ipo.get_ubx_relaxed(), dtype=np.float64)
        self.solver.iterative_refinement(mu, self.mult, rhs, self.vars, self.grad, lbx,
                                         ubx, self.px, self.res, self.ir_corr)
        ipo.compute_update(mu, self.vars, self.px, self.update)

    # -- barrier --------------------------------------------------------------------
    def _heuristic_mu(self, o):
        avg, xi = self.ipo.compute_complementarity(self.vars)
        r = o["heuristic_barrier_r"]
        f = min((1.0 - r) * (1.0 - xi) / xi, 2.0) ** 3 if xi > 1e-10 else 8.0
        floor = min(o["convergence_tolerance"], o["compl_inf_tol"]) / (o["barrier_tol_factor"] + 1.0)
        return max(o["heuristic_barrier_gamma"] * f * avg, floor)

    # -- filter line search -----------------------------------------------------------
    def _line_search(self, ax, az, filt, o, tau, phi0, wd_ref=None):
        """Returns (alpha / ax, trials, accepted, last rejection by the
        filter)."""
        ipo = self.ipo
        gt, gp = o["filter_gamma_theta"], o["filter_gamma_phi"]
        delta, s_t, s_p = o["filter_delta"], o["filter_s_theta"], o["filter_s_phi"]
        eta = o["filter_eta_phi"]
        eps10 = 10.0 * _EPS
        if wd_ref is not None:
            th0, ph0, dphi = wd_ref
        else:
            th0, ph0 = self._theta(), phi0
            dphi = ipo.compute_barrier_dphi(self.mu, self.vars, self.update, self.res,
                                            self.px, self.diag)
        t0 = self._theta0 if self._theta0 is not None else th0
        th_min, th_max = 1e-4 * max(1.0, t0), 1e4 * max(1.0, t0)
        if wd_ref is not None:
            a_min = ax
        else:
            a_min = gt
            if dphi < 0.0:
                a_min = min(gt, gp * th0 / -dphi)
                if th0 <= th_min:
                    a_min = min(a_min, delta * th0 ** s_t / (-dphi) ** s_p)
            a_min *= 0.05

        def f_type(a):
            return dphi < 0.0 and a * (-dphi) ** s_p > delta * th0 ** s_t

        def armijo(phi, a):
            return (phi - ph0) - eta * a * dphi <= eps10 * abs(ph0)

        def sufficient(phi, th):
            if phi > ph0:
                base = math.log10(abs(ph0)) if abs(ph0) > 10.0 else 1.0
                if math.log10(max(phi - ph0, 1e-300)) > 5.0 + base:
                    return False
            return (th - (1.0 - gt) * th0 <= eps10 * abs(th0)) or \
                ((phi - ph0) + gp * th0 <= eps10 * abs(ph0))

        def accept(phi, th, a):
            if th > th_max:
                return False, False
            if a > 0.0 and f_type(a) and th0 <= th_min:
                if not armijo(phi, a):
                    return False, False
            elif not sufficient(phi, th):
                return False, False
            ok = filt.acceptable(phi, th)
            return ok, not ok

        def record(phi, a):
            if not (f_type(a) and armijo(phi, a)):
                filt.add(ph0, th0)

        soc = o["second_order_correction"]
        if soc:
            ipo.compute_residual(self.mu, self.vars, self.grad, self.res)
            res0 = _copy(_a(self.res))
            upd0 = ipo.create_opt_vector()
            upd0.copy(self.update)
            px0 = _copy(_a(self.px))
        a = ax
        n = 0
        by_filter = False
        mm = None
        while a > a_min or n == 0:
            if n >= o["max_line_search_iterations"]:
                break
            ipo.apply_step_update(a, az, self.vars, self.update, self.temp)
            self._gradient(self._sol(self.temp))
            th = self._theta(self.temp)
            phi = self._barrier_objective(self.temp)
            ok, fr = accept(phi, th, a)
            if ok:
                record(phi, a)
                self.vars.copy(self.temp)
                return a / ax, n + 1, True, by_filter
            by_filter = fr
            if soc and n == 0 and th >= th0:
                # second-order corrections on the constraint residual
                c_soc = _copy(res0)
                if mm is None:
                    mm = InertiaCorrection._mask(self.mult, c_soc)
                a_soc, th_old, done = a, 0.0, False
                for k in range(o["filter_max_soc"]):
                    if k > 0 and th > o["filter_kappa_soc"] * th_old:
                        break
                    th_old = th
                    ipo.compute_residual(self.mu, self.temp, self.grad, self.res)
                    tr = _a(self.res)
                    c_soc[mm] = tr[mm] + a_soc * c_soc[mm]
                    tr[...] = c_soc
                    _sync(self.res)
                    self._gradient(self._sol())
                    try:
                        self.solver.solve(self.res, self.px)
                    except Exception:
                        break
                    ipo.compute_update(self.mu, self.vars, self.px, self.update)
                    sax, _, saz, _ = ipo.compute_max_step(tau, self.vars, self.update)
                    ipo.apply_step_update(sax, saz, self.vars, self.update, self.temp)
                    self._gradient(self._sol(self.temp))
                    th = self._theta(self.temp)
                    phi = self._barrier_objective(self.temp)
                    sok, _ = accept(phi, th, a)
                    if sok:
                        record(phi, a)
                        self.vars.copy(self.temp)
                        done = True
                        break
                    a_soc = sax
                if done:
                    return 1.0, n + 1, True, False
                self.update.copy(upd0)
                _a(self.px)[...] = px0
                _sync(self.px)
            a *= o["backtracking_factor"]
            n += 1
        self._gradient(self._sol())
        return a / ax, n, False, by_filter

    def _line_search_watchdog(self, ax, az, filt, o, tau, wd, factor_ok):
        ipo = self.ipo
        if wd.on and (not factor_ok or ax < 1e-16):
            self._restore(wd)
            wd.on, wd.shortened = False, 0
        if not wd.on and wd.trigger > 0 and wd.shortened >= wd.trigger:
            wd.x = _copy(_a(self._sol()))
            wd.upd.copy(self.update)
            wd.px = _copy(_a(self.px))
            wd.alpha = ax
            wd.theta = self._theta()
            wd.barr = self._barrier_objective(self.vars)
            wd.dphi = ipo.compute_barrier_dphi(self.mu, self.vars, self.update, self.res,
                                               self.px, self.diag)
            wd.on, wd.trials = True, 0
        phi0 = self._barrier_objective(self.vars)
        ref = (wd.theta, wd.barr, wd.dphi) if wd.on else None
        skip = False
        while True:
            out = self._line_search(ax, az, filt, o, tau, phi0, None if skip else ref)
            alpha, iters, ok, by_filter = out
            if wd.on and not skip:
                if ok:
                    wd.on, wd.shortened = False, 0
                    break
                wd.trials += 1
                if wd.trials > wd.max_trials:
                    self._restore(wd)
                    wd.on, wd.shortened = False, 0
                    ax, _, az, _ = ipo.compute_max_step(tau, self.vars, self.update)
                    phi0 = self._barrier_objective(self.vars)
                    skip = True
                    continue
                ok = True
                break
            break
        return alpha, iters, ok, by_filter

    def _restore(self, wd):
        xa = _a(self._sol())
        xa[...] = wd.x
        _sync(self._sol())
        self.update.copy(wd.upd)
        _a(self.px)[...] = wd.px
        _sync(self.px)
        self._gradient(self._sol())

    # -- restoration ----------------------------------------------------------------
    def _restoration(self, ic, filt, o, x):
        ipo = self.ipo
        tol = o["convergence_tolerance"]
        bt, mls = o["backtracking_factor"], o["max_line_search_iterations"]
        th_k = th_start = self._theta()
        th_min = 1e-4 * max(1.0, self._theta0 if self._theta0 is not None else th_k)
        if th_k < max(tol, th_min):
            # small theta: the filter blocks progress -- KKT-descent steps,
            # else reset the filter
            r0 = ipo.compute_residual(self.mu, self.vars, self.grad, self.res)
            tau = max(o["tau_min"], 1.0 - self.mu) if o["adaptive_tau"] else o["fraction_to_boundary"]
            ax, _, az, _ = ipo.compute_max_step(tau, self.vars, self.update)
            a = 1.0
            for _ in range(mls):
                ipo.apply_step_update(a * ax, az, self.vars, self.update, self.temp)
                self._gradient(self._sol(self.temp))
                r1 = ipo.compute_residual(self.mu, self.temp, self.grad, self.res)
                if r1 < r0:
                    phi = self._barrier_objective(self.temp)
                    th = self._theta(self.temp)
                    if filt.acceptable(phi, th):
                        self.vars.copy(self.temp)
                        return True
                    if r1 < 0.99 * r0:
                        self.vars.copy(self.temp)
                        filt.clear()
                        self._theta0 = th
                        return True
                a *= bt
            self._gradient(self._sol())
            filt.clear()
            self._theta0 = th_k
            return True
        # large theta: Newton steps at a raised barrier aimed at a 10%
        # reduction of the constraint violation
        filt.add(self._barrier_objective(self.vars), th_k)
        target = 0.9 * th_k
        saved = self.mu
        levels = sorted({m for m in (max(saved, 1e-2), 0.1, 1.0) if m >= saved})
        per = max(3, o["filter_restoration_max_iter"] // len(levels))
        for mu_r in levels:
            self.mu = mu_r
            ic.mu = mu_r
            for _ in range(per):
                xv = self._sol()
                self._gradient(xv)
                ipo.compute_diagonal(self.vars, self.diag)
                dr = _copy(_a(self.diag))
                self._direction(xv, dr, ic, o)
                tau = max(o["tau_min"], 1.0 - mu_r) if o["adaptive_tau"] else o["fraction_to_boundary"]
                ax, _, az, _ = ipo.compute_max_step(tau, self.vars, self.update)
                a, took = 1.0, False
                for _ in range(mls):
                    ipo.apply_step_update(a * ax, a * az, self.vars, self.update, self.temp)
                    self._gradient(self._sol(self.temp))
                    th = self._theta(self.temp)
                    if th < th_k:
                        self.vars.copy(self.temp)
                        th_k, took = th, True
                        break
                    a *= bt
                if not took or th_k < target:
                    break
            if th_k < target:
                break
        self.mu = saved
        ic.mu = saved
        self._gradient(self._sol())
        ipo.compute_diagonal(self.vars, self.diag)
        return th_k < 0.99 * th_start

    # -- safeguards -------------------------------------------------------------------
    def _floor_slacks(self, mu):
        """Floor the stored slacks at eps min(1, mu) (bound_safeguards.py:
        17-82); x moves with them.  Returns the number adjusted."""
        ipo = self.ipo
        s_min = _EPS * min(1.0, mu)
        if s_min == 0.0:
            s_min = np.finfo(np.float64).tiny
        sl = np.asarray(self.vars.get_sl(), dtype=np.float64)
        su = np.asarray(self.vars.get_su(), dtype=np.float64)
        if not ((sl.size and sl[self._fl].min(initial=np.inf) < s_min) or
                (su.size and su[self._fu].min(initial=np.inf) < s_min)):
            return 0
        zl = np.asarray(self.vars.get_zl(), dtype=np.float64)
        zu = np.asarray(self.vars.get_zu(), dtype=np.float64)
        move = 1.81898940354586e-12
        n = 0
        for s, z, fin, b in ((sl, zl, self._fl, self._lbx), (su, zu, self._fu, self._ubx)):
            small = fin & (s < s_min)
            if small.any():
                idx = np.nonzero(small)[0]
                g = np.maximum(s[idx], 0.0)
                zz = np.maximum(z[idx], np.finfo(np.float64).tiny)
                s[idx] = np.minimum(np.maximum(mu / zz, s_min),
                                    move * np.maximum(1.0, np.abs(b[idx])) + g)
                n += len(idx)
        self._set_slacks(sl, su)
        return n

    def _set_slacks(self, sl, su):
        v = self.vars
        npr = len(sl)
        xa = _a(v.get_solution())
        lb, ub = self._lbx, self._ubx
        newx = _host(xa).copy()
        pi = self._pidx
        for i in np.nonzero(self._fl)[0]:
            newx[pi[i]] = lb[i] + sl[i]
        for i in np.nonzero(self._fu)[0]:
            newx[pi[i]] = ub[i] - su[i]
        if hasattr(v, "slacks") and not hasattr(v, "tup"):       # device OptVector
            v.slacks[:npr] = torch.as_tensor(sl, device=v.slacks.device)
            v.slacks[npr:] = torch.as_tensor(su, device=v.slacks.device)
            xa.copy_(torch.as_tensor(newx, device=xa.device))
        else:
            sv = v.get_slacks()
            arr = _a(sv)
            arr[:npr], arr[npr:] = sl, su
            _sync(sv)
            xa[...] = newx
            _sync(v.get_solution())

    # -- convergence -------------------------------------------------------------------
    def _check(self, i, o, res_norm, st):
        err, d, p, c = self._kkt_error()
        if err <= o["convergence_tolerance"] and d <= o["dual_inf_tol"] and \
                p <= o["constr_viol_tol"] and c <= o["compl_inf_tol"]:
            return CONVERGED
        xmax = float(np.abs(_host(_a(self._sol()))).max())
        if xmax > o["diverging_iterates_tol"]:
            return DIVERGED
        ok = (err <= o["acceptable_tol"] and d <= o["acceptable_dual_inf_tol"] and
              p <= o["acceptable_constr_viol_tol"] and c <= o["acceptable_compl_inf_tol"])
        if o["acceptable_iter"] > 0 and ok:
            st["acc"] += 1
            if st["acc"] >= o["acceptable_iter"]:
                return ACCEPTABLE
        else:
            st["acc"] = 0
        rel = abs(res_norm - st["prev_res"]) / max(res_norm, 1e-30)
        st["floor"] = st["floor"] + 1 if (rel < 1e-14 and i > 0) else 0
        if st["floor"] >= 3 and ok:
            return FLOOR
        return CONTINUE

    # -- main loop ------------------------------------------------------------------------
    def optimize(self, options=None):
        """Run the interior-point iteration; returns a dict like amigo's:
        converged, iterations (a record per iteration: residual,
        barrier_param, step lengths, line-search trials, inertia
        perturbation, KKT error components, barrier objective), plus
        the final objective-free summary fields and the wall time.
        Options are amigo's (amigo/algorithm/default_options.py): an
        unknown name is a ValueError as there; a name of amigo's whose
        value selects a strategy other than its default algorithm raises
        NotImplementedError."""
        o = dict(DEFAULT_OPTIONS)
        for k, v in (options or {}).items():
            if k in o:
                o[k] = v
            elif k in DEFAULT_ALGORITHM_OPTIONS:
                if k not in DIAGNOSTIC_OPTIONS and v != DEFAULT_ALGORITHM_OPTIONS[k]:
                    raise NotImplementedError(
                        "option %s=%r selects a part of amigo's optimizer other than "
                        "its default algorithm, which is the one restated here" % (k, v))
            else:
                raise ValueError("Unrecognized option %s" % k)
        t0 = time.perf_counter()
        ipo = self.ipo
        self.mu = o["initial_barrier_param"]
        self._initialize(o)
        lbx = np.asarray(ipo.get_lbx(), dtype=np.float64)
        ubx = np.asarray(ipo.get_ubx(), dtype=np.float64)
        self._lbx, self._ubx = lbx, ubx
        self._fl, self._fu = np.isfinite(lbx), np.isfinite(ubx)
        self._nbounds = int(self._fl.sum() + self._fu.sum())
        self._pidx = np.nonzero(~self.mult)[0]
        ic = InertiaCorrection(self.mult, self.mu)
        filt = _Filter(o["filter_gamma_phi"], o["filter_gamma_theta"])
        self._theta0 = None
        wd = _Watchdog(ipo, o["watchdog_shortened_iter_trigger"], o["watchdog_trial_iter_max"])
        st = dict(line=0, ax=0.0, az=0.0, prev_res=float("inf"), acc=0, floor=0, rej=0,
                  filt_rej=0, resets=0)
        records = []
        out = dict(converged=False)
        x = self._sol()
        tol = o["convergence_tolerance"]
        for i in range(o["max_iterations"]):
            res_norm = ipo.compute_residual(self.mu, self.vars, self.grad, self.res)
            ic.mu = self.mu
            if self._theta0 is None:
                self._theta0 = self._theta()
            err, d_inf, p_inf, c_inf = self._kkt_error()
            records.append(dict(iteration=i, residual=res_norm, barrier_param=self.mu,
                                line_iters=st["line"], alpha_x=st["ax"], alpha_z=st["az"],
                                inertia_delta=ic.last_delta_w, inf_pr=p_inf, inf_du=d_inf,
                                compl=c_inf, nlp_error=err,
                                objective=self._barrier_objective(self.vars)))
            status = self._check(i, o, res_norm, st)
            if status in (CONVERGED, ACCEPTABLE, FLOOR):
                out.update(converged=True, acceptable=status != CONVERGED)
                break
            if status == DIVERGED:
                break
            st["prev_res"] = res_norm
            rejected = False
            ipo.compute_diagonal(self.vars, self.diag)
            diag_base = _copy(_a(self.diag))
            mu_before = self.mu
            if i > 0 and self.mu > min(tol, o["compl_inf_tol"]) / (o["barrier_tol_factor"] + 1.0):
                self.mu = self._heuristic_mu(o)
            ic.mu = self.mu
            factor_ok = self._direction(x, diag_base, ic, o)
            if self.mu != mu_before:
                ic.mu = self.mu
                filt.clear()
                self._theta0 = self._theta()
                wd.reset()
                st["filt_rej"] = st["resets"] = 0
            if not factor_ok:
                st["rej"] += 1
                self.mu = mu_before
                st["line"], st["ax"], st["az"] = 0, 0.0, 0.0
                st["rej"] = self._raise_mu(st["rej"], o)
                continue
            ipo.compute_residual(self.mu, self.vars, self.grad, self.res)
            tau = max(o["tau_min"], 1.0 - self.mu) if o["adaptive_tau"] else o["fraction_to_boundary"]
            ax, _, az, _ = ipo.compute_max_step(tau, self.vars, self.update)
            alpha, st["line"], ok, by_filter = self._line_search_watchdog(
                ax, az, filt, o, tau, wd, factor_ok)
            if ok:
                st["filt_rej"] = st["filt_rej"] + 1 if by_filter else 0
                if st["filt_rej"] >= o["filter_reset_trigger"] and \
                        st["resets"] < o["max_filter_resets"]:
                    filt.clear()
                    st["resets"] += 1
                    st["filt_rej"] = 0
            else:
                if self._restoration(ic, filt, o, x):
                    ok = True
                    st["line"] = 0
                    wd.shortened = 0
                else:
                    rejected = True
                    st["rej"] += 1
            if ok:
                self._floor_slacks(self.mu)
                ipo.reset_bound_multipliers(self.mu, 1e10, self.vars)
                self._gradient(self._sol())
            if rejected:
                st["ax"] = st["az"] = 0.0
                self.mu = mu_before
                st["rej"] = self._raise_mu(st["rej"], o)
            else:
                st["ax"], st["az"] = alpha * ax, az
                st["rej"] = 0
                if not wd.on:
                    wd.shortened = 0 if (alpha == 1.0 or st["line"] == 1) else wd.shortened + 1
        out.update(iterations=records, time_s=time.perf_counter() - t0)
        return out

    def _raise_mu(self, rej, o):
        if rej >= o["max_consecutive_rejections"]:
            new = min(self.mu * o["barrier_increase_factor"], o["initial_barrier_param"])
            if new > self.mu:
                self.mu = new
            return 0
        return rej

    def get_solution(self):
        return self._sol()
