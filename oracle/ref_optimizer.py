"""Run the reference's own interior-point driver on the host (test
infrastructure only; needs the reference sources, so it runs where they are
present and is used to generate committed golden data).

The reference's `Optimizer` (amigo/algorithm/ipm_driver.py:109-483 and the
modules it composes) is pure Python over three interfaces: the compiled
`InteriorPointOptimizer` backend (amigo/amigo.cpp:747-907 over
include/interior_point_optimizer.h), a linear solver (here its own
`AmigoSolver`, amigo/algorithm/solvers/amigo_solver.py, over the compiled
`SparseLDL`) and the problem (`OptimizationProblem`: create_vector,
create_matrix, gradient, hessian, add_diagonal).  The compiled module
cannot be built here (its generated component code needs A2D), so a
stand-in `amigo.amigo` module is installed in its place:
  * `InteriorPointOptimizer` calls the reference's own interior_point_
    backend.h functions (oracle/_ref), with the class's glue
    (interior_point_optimizer.h:114-598: index split, relaxed bounds,
    NLP scaling, slack mapping) restated in numpy;
  * `SparseLDL` is the reference's SparseLDL (oracle/_ref);
  * the problem evaluates the model's derivatives with the numpy
    restatement in oracle/ (cartpole_oracle.py).
The driver code itself is imported unchanged from the reference tree.
"""
import enum
import importlib
import os
import sys
import types

import numpy as np

from . import ref

REF_ROOT = os.environ.get("AMIGO_REF_ROOT", "/root/reference")


class HostVector:
    """amigo.Vector on the host (HOST_ONLY): get_array is a view."""

    def __init__(self, n=0, arr=None):
        self.arr = np.zeros(int(n)) if arr is None else np.asarray(arr, dtype=np.float64)

    def get_array(self):
        return self.arr

    def get_size(self):
        return len(self.arr)

    def __len__(self):
        return len(self.arr)

    def copy_host_to_device(self):
        pass

    def copy_device_to_host(self):
        pass

    def zero(self):
        self.arr[:] = 0.0

    def copy(self, other):
        self.arr[:] = other.arr


class HostCSRMat:
    def __init__(self, n, rowp, cols, diag_pos):
        self.n = n
        self.rowp = np.asarray(rowp, np.int32)
        self.cols = np.asarray(cols, np.int32)
        self.data = np.zeros(int(self.rowp[-1]))
        self.diag_pos = diag_pos

    def get_nonzero_structure(self):
        return self.n, self.n, len(self.data), self.rowp, self.cols

    def get_data(self):
        return self.data

    def copy_data_device_to_host(self):
        pass

    def copy_data_host_to_device(self):
        pass


class HostOptVector:
    def __init__(self, npr, x):
        self.x = x
        self.duals = np.zeros(2 * npr)
        self.slacks = np.zeros(2 * npr)
        self.np = npr

    def get_solution(self):
        return self.x

    def tup(self):
        n = self.np
        return (self.x.arr, self.duals[:n], self.duals[n:], self.slacks[:n], self.slacks[n:])

    # copies as lists, as the compiled binding returns them
    def get_zl(self):
        return list(self.duals[:self.np])

    def get_zu(self):
        return list(self.duals[self.np:])

    def get_sl(self):
        return list(self.slacks[:self.np])

    def get_su(self):
        return list(self.slacks[self.np:])

    def copy(self, other):
        self.x.arr[:] = other.x.arr
        self.duals[:] = other.duals
        self.slacks[:] = other.slacks

    def get_slacks(self):
        return HostVector(arr=self.slacks)

    def copy_host_to_device(self):
        pass

    def copy_device_to_host(self):
        pass

    def zero(self):
        self.x.arr[:] = 0.0
        self.duals[:] = 0.0
        self.slacks[:] = 0.0


class HostProblem:
    """OptimizationProblem over a model's numpy derivatives: `deriv` gives
    gradient(x, alpha) and hessian_values(x, alpha) on model.rowp/cols."""

    def __init__(self, model, gradient, hessian_values, lagrangian):
        self.m = model
        self._g = gradient
        self._h = hessian_values
        self._l = lagrangian
        self.mult = np.asarray(model.mult, bool)

    def get_multiplier_indicator(self):
        return self.mult.astype(np.int32)

    def get_num_variables(self):
        return self.m.n

    def create_vector(self):
        return HostVector(self.m.n)

    def create_matrix(self, loc=None):
        return HostCSRMat(self.m.n, self.m.rowp, self.m.cols, self.m.diag_pos)

    def gradient(self, alpha, x, g):
        g.arr[:] = self._g(x.arr, alpha)

    def hessian(self, alpha, x, hess):
        hess.data[:] = self._h(x.arr, alpha)

    def add_diagonal(self, diag, hess):
        hess.data[self.m.diag_pos] += diag.arr

    def lagrangian(self, alpha, x):
        return float(self._l(x.arr, alpha))

    def get_data_vector(self):
        return HostVector(0)

    def update(self, x):
        pass


class InteriorPointOptimizer:
    """The reference backend class, its glue restated over the reference's
    interior_point_backend.h functions (oracle/_ref)."""

    def __init__(self, problem, lower, upper):
        self.problem = problem
        mult = np.asarray(problem.get_multiplier_indicator(), bool)
        lb, ub = lower.arr, upper.arr
        self.n = len(mult)
        self.pidx = np.nonzero(~mult)[0].astype(np.int32)
        self.cidx = np.nonzero(mult)[0].astype(np.int32)
        self.np_, self.nc_ = len(self.pidx), len(self.cidx)
        self.lbx = lb[self.pidx].copy()
        self.ubx = ub[self.pidx].copy()
        self.lbh = lb[self.cidx].copy()
        self.lbx_r, self.ubx_r = None, None
        self.nslack = 0
        self.obj_scale = 1.0
        self.scaling = False
        self._ipm()

    def _ipm(self):
        lbx = self.lbx_r if self.lbx_r is not None else self.lbx
        ubx = self.ubx_r if self.ubx_r is not None else self.ubx
        self.R = ref.RefIPM(self.pidx, self.cidx, lbx, ubx, self.lbh)

    def create_opt_vector(self, x=None):
        return HostOptVector(self.np_, x if x is not None else self.problem.create_vector())

    def set_multipliers_value(self, v, x):
        x.arr[self.cidx] = v

    def set_design_vars_value(self, v, x):
        x.arr[self.pidx] = v

    def copy_multipliers(self, d, s):
        d.arr[self.cidx] = s.arr[self.cidx]

    def copy_design_vars(self, d, s):
        d.arr[self.pidx] = s.arr[self.pidx]

    def initialize_multipliers_and_slacks(self, mu, grad, vars):
        R = self.R
        x, zl, zu, sl, su = vars.tup()
        lib = ref.lib()
        lib.ref_ipm_initialize(self.np_, self.nc_, ref._ptr(R.pidx, "i"), ref._ptr(R.cidx, "i"),
                               ref._ptr(R.lbx, "d"), ref._ptr(R.ubx, "d"), ref._ptr(R.lbh, "d"),
                               ref._d(mu), ref._ptr(x, "d"), ref._ptr(zl, "d"),
                               ref._ptr(zu, "d"), ref._ptr(sl, "d"), ref._ptr(su, "d"))

    def compute_residual(self, mu, vars, grad, res):
        res.arr[:] = self.R.compute_residual(mu, vars.tup(), grad.arr)
        return float(np.sqrt(res.arr @ res.arr))

    def compute_residual_and_infeasibility(self, mu, vars, grad, res):
        R = self.R
        g = np.ascontiguousarray(grad.arr)
        out = np.zeros(self.n)
        d, p = ref.ctypes.c_double(), ref.ctypes.c_double()
        ref.lib().ref_ipm_compute_residual_and_infeasibility(
            ref._d(mu), *R._args(*vars.tup()), ref._ptr(g, "d"), ref._ptr(out, "d"),
            ref.ctypes.byref(d), ref.ctypes.byref(p))
        res.arr[:] = out
        return d.value, p.value

    def compute_diagonal(self, vars, diag):
        diag.arr[:] = self.R.compute_diagonal(vars.tup(), self.n)

    def compute_update(self, mu, vars, px, upd):
        upd.x.arr[:] = px.arr
        dzl, dzu = self.R.compute_bound_dual_step(mu, vars.tup(), px.arr)
        upd.duals[:self.np_] = dzl
        upd.duals[self.np_:] = dzu

    def compute_max_step(self, tau, vars, upd):
        return self.R.compute_max_step(tau, vars.tup(), upd.x.arr, upd.duals[:self.np_],
                                       upd.duals[self.np_:])

    def apply_step_update(self, ax, az, vars, upd, tmp):
        out = self.R.apply_step(ax, az, vars.tup(), upd.x.arr, upd.duals[:self.np_],
                                upd.duals[self.np_:])
        tmp.x.arr[:] = out[0]
        tmp.duals[:self.np_], tmp.duals[self.np_:] = out[1], out[2]
        tmp.slacks[:self.np_], tmp.slacks[self.np_:] = out[3], out[4]

    def compute_complementarity(self, vars):
        s0, s1, mn = self.R.compute_complementarity(vars.tup())
        avg = s0 / s1 if s1 > 0 else 0.0
        gm = mn if np.isfinite(mn) else np.finfo(np.float64).max
        xi = max(0.0, min(1.0, gm / avg)) if avg > 0 else 1.0
        return avg, xi

    def compute_complementarity_sq(self, vars):
        return self.R.compute_complementarity_sq(vars.tup(), 0.0)

    def compute_max_comp_deviation(self, vars, mu):
        return self.R.compute_max_comp_deviation(vars.tup(), mu)

    def compute_kkt_error(self, vars, grad):
        R = self.R
        g = np.ascontiguousarray(grad.arr)
        d, p, c = ref.ctypes.c_double(), ref.ctypes.c_double(), ref.ctypes.c_double()
        ref.lib().ref_ipm_compute_kkt_error_sq(*R._args(*vars.tup()), ref._ptr(g, "d"),
                                               ref.ctypes.byref(d), ref.ctypes.byref(p),
                                               ref.ctypes.byref(c))
        return d.value, p.value, c.value

    def compute_kkt_error_mu(self, mu, vars, grad):
        return self.R.compute_kkt_error(mu, vars.tup(), grad.arr)

    def compute_constraint_violation_1norm(self, vars, grad):
        return self.R.compute_constraint_violation_1norm(vars.tup(), grad.arr)

    def compute_barrier_log_sum(self, barrier_param, vars):
        return self.R.compute_barrier_log_sum(barrier_param, vars.tup())

    def compute_barrier_dphi_direct(self, barrier_param, vars, grad, px):
        return self.R.compute_barrier_dphi(barrier_param, vars.tup(), grad.arr, px.arr)

    def compute_barrier_dphi(self, barrier_param, vars, update, res, px, diag):
        R = self.R
        r, p_, d = (np.ascontiguousarray(a.arr) for a in (res, px, diag))
        return ref.lib().ref_ipm_compute_barrier_dphi_from_kkt(
            *R._args(*vars.tup()), ref._ptr(r, "d"), ref._ptr(p_, "d"), ref._ptr(d, "d"))

    def reset_bound_multipliers(self, barrier_param, kappa_sigma, vars):
        zl, zu = self.R.reset_bound_multipliers(barrier_param, kappa_sigma, vars.tup())
        vars.duals[:self.np_], vars.duals[self.np_:] = zl, zu

    def compute_affine_start_point(self, beta_min, vars, upd, dst):
        zl, zu = self.R.compute_affine_start_point(beta_min, vars.tup(), upd.duals[:self.np_],
                                                   upd.duals[self.np_:])
        dst.duals[:self.np_], dst.duals[self.np_:] = zl, zu

    def compute_dual_residual_vector(self, vars, grad, output):
        R = self.R
        g = np.ascontiguousarray(grad.arr)
        out = np.zeros(len(output.arr))
        ref.lib().ref_ipm_compute_dual_residual_vector(*R._args(*vars.tup()), ref._ptr(g, "d"),
                                                       ref._ptr(out, "d"), len(out))
        output.arr[:] = out

    def get_kkt_element_counts(self):
        nc = int(np.sum(~np.isinf(self.lbx)) + np.sum(~np.isinf(self.ubx)))
        return self.np_, self.nc_, nc

    def check_update(self, *args):
        return None

    def get_lbx(self):
        return list(self.lbx)

    def get_ubx(self):
        return list(self.ubx)

    def get_lbx_relaxed(self):
        return list(self.lbx_r if self.lbx_r is not None else self.lbx)

    def get_ubx_relaxed(self):
        return list(self.ubx_r if self.ubx_r is not None else self.ubx)

    def get_num_inequalities(self):
        return 0

    def get_num_design_variables(self):
        return self.np_

    def relax_bounds(self, factor=1e-8, constr_viol_tol=1e-4):
        if factor <= 0:
            return
        lo, hi = np.zeros(self.np_), np.zeros(self.np_)
        R = ref.RefIPM(self.pidx, self.cidx, self.lbx, self.ubx, self.lbh)
        ref.lib().ref_ipm_relax_bounds(self.np_, self.nc_, ref._ptr(R.pidx, "i"),
                                       ref._ptr(R.cidx, "i"), ref._ptr(R.lbx, "d"),
                                       ref._ptr(R.ubx, "d"), ref._ptr(R.lbh, "d"),
                                       ref._ptr(lo, "d"), ref._ptr(hi, "d"),
                                       ref._d(factor), ref._d(constr_viol_tol))
        self.lbx_r, self.ubx_r = lo, hi
        self._ipm()

    def set_slack_mapping(self, slack_indices, constr_indices):
        self.sidx = np.asarray(slack_indices, np.int32)
        self.scidx = np.asarray(constr_indices, np.int32)
        self.nslack = len(self.sidx)

    def initialize_slacks(self, grad, vars):
        for si, ci in zip(getattr(self, "sidx", []), getattr(self, "scidx", [])):
            vars.x.arr[si] = grad.arr[ci] + vars.x.arr[si]

    def has_slacks(self):
        return self.nslack > 0

    def compute_nlp_scaling(self, x, grad, max_gradient=100.0, min_value=1e-8):
        g = grad.arr
        gmax = float(np.max(np.abs(g[self.pidx]))) if self.np_ else 0.0
        self.obj_scale = max_gradient / gmax if gmax > max_gradient else 1.0
        self.obj_scale = max(self.obj_scale, min_value)
        H = self.problem.create_matrix()
        self.problem.hessian(1.0, x, H)
        self.dc = np.ones(self.nc_)
        for j, row in enumerate(self.cidx):
            a, b = H.rowp[row], H.rowp[row + 1]
            rm = float(np.max(np.abs(H.data[a:b]))) if b > a else 0.0
            dc = max_gradient / rm if rm > max_gradient else 1.0
            self.dc[j] = max(dc, min_value)
        for j in range(self.nc_):
            if self.dc[j] != 1.0:
                self.lbh[j] *= self.dc[j]
        self.svec = np.ones(self.n)
        self.svec[self.cidx] = self.dc
        self.scaling = True
        self._ipm()

    def apply_gradient_scaling(self, grad):
        if self.scaling:
            grad.arr[self.cidx] *= self.dc

    def apply_hessian_scaling(self, hess):
        if self.scaling:
            rows = np.repeat(np.arange(self.n), np.diff(hess.rowp))
            hess.data *= self.svec[rows] * self.svec[hess.cols]

    def scale_multipliers(self, x):
        if self.scaling:
            x.arr[self.cidx] *= self.dc

    def unscale_multipliers(self, x):
        if self.scaling:
            x.arr[self.cidx] /= self.dc

    def get_obj_scale(self):
        return self.obj_scale

    def has_scaling(self):
        return self.scaling


class SparseLDL:
    """amigo.SparseLDL: the reference's own SparseLDL (oracle/_ref)."""

    def __init__(self, mat, solver_type=0, ustab=0.01, pivot_tol=1e-14,
                 delay_growth=2.0, order=1):
        self.mat = mat
        self.R = ref.RefSparseLDL(mat.n, mat.rowp, mat.cols, order="AMD",
                                  ustab=ustab, pivot_tol=pivot_tol)

    def factor(self):
        self.R.factor(self.mat.data)
        return 0

    def solve(self, x):
        arr = x.arr if isinstance(x, HostVector) else x
        arr[:] = self.R.solve(arr)

    def get_inertia(self):
        return self.R.inertia()


def install():
    """Put the stand-in compiled module and the reference's Python package
    (its __init__ skipped: it imports the compiled module's full surface)
    into sys.modules; returns amigo.algorithm."""
    if not os.path.isdir(os.path.join(REF_ROOT, "amigo", "algorithm")):
        raise RuntimeError("reference sources not found")
    if "amigo.algorithm" in sys.modules and getattr(sys.modules["amigo"], "_oracle_stub", False):
        return sys.modules["amigo.algorithm"]
    pkg = types.ModuleType("amigo")
    pkg.__path__ = [os.path.join(REF_ROOT, "amigo")]
    pkg._oracle_stub = True
    core = types.ModuleType("amigo.amigo")

    class OrderingType(enum.IntEnum):
        NESTED_DISSECTION = 0
        AMD = 1
        MULTI_COLOR = 2
        NATURAL = 3
        DEFAULT = 1

    class SolverType(enum.IntEnum):
        LDL = 0
        CHOLESKY = 1

    class MemoryLocation(enum.IntEnum):
        HOST_ONLY = 0
        DEVICE_ONLY = 1
        HOST_AND_DEVICE = 2

    class _Unavailable:
        def __init__(self, *a, **k):
            raise RuntimeError("not provided by the oracle stand-in")

    for name, obj in dict(OrderingType=OrderingType, SolverType=SolverType,
                          MemoryLocation=MemoryLocation, Vector=HostVector,
                          CSRMat=HostCSRMat, SparseLDL=SparseLDL,
                          InteriorPointOptimizer=InteriorPointOptimizer).items():
        setattr(core, name, obj)
        setattr(pkg, name, obj)
    for name in ("reorder_model", "VectorInt", "OptimizationProblem", "AliasTracker",
                 "NodeOwners", "ExternalComponentGroup", "SlackComponent",
                 "SparseCholesky"):
        setattr(core, name, _Unavailable)
        setattr(pkg, name, _Unavailable)
    sys.modules["amigo"] = pkg
    sys.modules["amigo.amigo"] = core
    return importlib.import_module("amigo.algorithm")


class HostModel:
    """The Model surface the Optimizer touches: its problem and no slacks."""

    def __init__(self, problem):
        self._p = problem
        self.num_slacks = 0

    def get_problem(self):
        return self._p


def optimize(m, gradient, hessian_values, lagrangian, objective, options=None, quiet=True):
    """Run the reference Optimizer with its AmigoSolver on the model `m`
    (n, mult, lower, upper, x0, rowp, cols, diag_pos); returns a dict with
    the iteration records, convergence flag, final x, objective and the
    final KKT error (max of the scaled infinity norms the driver reports)."""
    alg = install()
    P = HostProblem(m, gradient, hessian_values, lagrangian)
    model = HostModel(P)
    x = HostVector(arr=np.array(m.x0, dtype=np.float64))
    lo = HostVector(arr=np.array(m.lower, dtype=np.float64))
    hi = HostVector(arr=np.array(m.upper, dtype=np.float64))
    opt = alg.Optimizer(model, x, lo, hi, solver="amigo")
    import contextlib
    import io
    sink = io.StringIO()
    with (contextlib.redirect_stdout(sink) if quiet else contextlib.nullcontext()):
        data = opt.optimize(dict(options or {}))
    xs = opt.vars.get_solution().arr.copy()
    return dict(converged=bool(data["converged"]), iterations=len(data["iterations"]) - 1,
                records=data["iterations"], x=xs, objective=float(objective(xs)),
                log=sink.getvalue())
