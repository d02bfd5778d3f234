"""InteriorPointOptimizer / OptVector with amigo's Python-visible API.

Mirrors the methods and return tuples that amigo's pybind module binds
(amigo/amigo.cpp:747-907) over include/interior_point_optimizer.h, with all
vector work in libamigo_b200.so's device kernels.  The iterate lives in HBM
as torch tensors; methods that return scalars synchronise once to read them.

The problem is described as amigo describes it: an n-vector in which every
entry is either a bounded primal (design variable or slack) or an equality
multiplier, a multiplier indicator, and lower/upper arrays (for multipliers
the lower array holds the constraint target lbh).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .linalg import Vector, _device, _stream_ptr


class OptVector:
    """Iterate storage (include/interior_point_optimizer.h:21-90):
    x (n: primals and multipliers), bound duals [zl | zu] and bound slacks
    [sl | su] (np each)."""

    def __init__(self, n, npr, device, x=None):
        self.n, self.np = n, npr
        self.device = device
        self.x = (torch.zeros(n, dtype=torch.float64, device=device)
                  if x is None else x)
        self.duals = torch.zeros(2 * npr, dtype=torch.float64, device=device)
        self.slacks = torch.ones(2 * npr, dtype=torch.float64, device=device)

    @property
    def zl(self):
        return self.duals[: self.np]

    @property
    def zu(self):
        return self.duals[self.np:]

    @property
    def sl(self):
        return self.slacks[: self.np]

    @property
    def su(self):
        return self.slacks[self.np:]

    def get_solution(self):
        return self.x

    def get_zl(self):
        return self.zl.cpu().numpy()

    def get_zu(self):
        return self.zu.cpu().numpy()

    def get_sl(self):
        return self.sl.cpu().numpy()

    def get_su(self):
        return self.su.cpu().numpy()

    def copy(self, other):
        self.x.copy_(other.x)
        self.duals.copy_(other.duals)
        self.slacks.copy_(other.slacks)


def _dev(v):
    if isinstance(v, Vector):
        return v.dev
    if isinstance(v, OptVector):
        return v.x
    return v


def _host(v):
    """numpy view of an array-like, a Vector's host array or a tensor."""
    if isinstance(v, Vector):
        return v.get_array()
    if isinstance(v, torch.Tensor):
        return v.cpu().numpy()
    if hasattr(v, "get_array"):
        return v.get_array()
    return v


class InteriorPointOptimizer:
    """Device IPM vector operations over a fixed primal/multiplier split.

    InteriorPointOptimizer(mult_indicator, lower, upper, device=None)
    matches the reference constructor's effect
    (include/interior_point_optimizer.h:114-166): primal entries keep
    [lower, upper] as bounds, multiplier entries take lower as lbh.
    """

    def __init__(self, problem, lower, upper, device=None):
        """problem: the reference's first argument, an object with
        get_multiplier_indicator() (and, for compute_nlp_scaling,
        create_matrix() / hessian(alpha, x, hess)), or the multiplier
        indicator itself; lower / upper: arrays or Vector objects."""
        self.device = _device(device)
        if hasattr(problem, "get_multiplier_indicator"):
            self.problem = problem
            mult = problem.get_multiplier_indicator()
        else:
            self.problem = None
            mult = problem
        mult = np.asarray(_host(mult)).astype(bool)
        lower = np.asarray(_host(lower), dtype=np.float64)
        upper = np.asarray(_host(upper), dtype=np.float64)
        self.n = len(mult)
        pidx = np.nonzero(~mult)[0].astype(np.int32)
        cidx = np.nonzero(mult)[0].astype(np.int32)
        self.np_, self.nc_ = len(pidx), len(cidx)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.pidx, self.cidx = t(pidx), t(cidx)
        self.lbx, self.ubx = t(lower[pidx]), t(upper[pidx])
        self.lbh = t(lower[cidx])
        # the unrelaxed bounds (get_lbx / get_ubx); relax_bounds moves
        # self.lbx / self.ubx, which the kernels use
        self.lbx0, self.ubx0 = self.lbx.clone(), self.ubx.clone()
        self._relaxed = False
        self._host_bounds = {}
        self._nslack = 0
        self._obj_scale = 1.0
        self._scaling = False
        self._dc = None
        self._scale = None
        self._out = torch.zeros(16, dtype=torch.float64, device=self.device)
        self._iout = torch.zeros(4, dtype=torch.int32, device=self.device)
        self._p = _lib.IpmProblem(self.n, self.np_, self.nc_,
                                  self.pidx.data_ptr(), self.cidx.data_ptr(),
                                  self.lbx.data_ptr(), self.ubx.data_ptr(),
                                  self.lbh.data_ptr())

    # -- helpers ---------------------------------------------------------
    def _s(self):
        return _stream_ptr(self.device)

    def _state(self, v):
        return _lib.IpmState(v.x.data_ptr(), v.zl.data_ptr(), v.zu.data_ptr(),
                             v.sl.data_ptr(), v.su.data_ptr())

    def _c(self, name, *args):
        return _lib.call(name, ctypes.byref(self._p), *args)

    # -- factories -------------------------------------------------------
    def create_opt_vector(self, x=None):
        xd = None if x is None else _dev(x)
        return OptVector(self.n, self.np_, self.device, xd)

    def get_num_design_variables(self):
        return self.np_

    def get_num_constraints(self):
        return self.nc_

    def get_num_equalities(self):
        return self.nc_

    def get_num_inequalities(self):
        return 0

    def _host_bound(self, name):
        """Host copy of a bound vector (numpy, n_primal), as the reference's
        bindings return them (amigo/amigo.cpp:853-880); cached until
        relax_bounds changes the relaxed ones."""
        c = self._host_bounds.get(name)
        if c is None:
            c = getattr(self, name).cpu().numpy()
            c.setflags(write=False)
            self._host_bounds[name] = c
        return c

    def get_lbx(self):
        """Primal lower bounds as given."""
        return self._host_bound("lbx0")

    def get_ubx(self):
        return self._host_bound("ubx0")

    def get_lbx_relaxed(self):
        """The bounds the IPM kernels use: relaxed once relax_bounds ran."""
        return self._host_bound("lbx" if self._relaxed else "lbx0")

    def get_ubx_relaxed(self):
        return self._host_bound("ubx" if self._relaxed else "ubx0")

    def get_kkt_element_counts(self):
        """(n_d, n_p, n_c): dual-stationarity rows, primal-feasibility rows
        and finite bounds (interior_point_optimizer.h:441-449)."""
        n_c = int(np.isfinite(self.get_lbx()).sum() + np.isfinite(self.get_ubx()).sum())
        return self.np_, self.nc_, n_c

    # -- setup -----------------------------------------------------------
    def relax_bounds(self, factor=1e-8, constr_viol_tol=1e-4):
        if factor <= 0:
            return
        _lib.call("ab_ipm_relax_bounds", self.np_, self.lbx0.data_ptr(),
                  self.ubx0.data_ptr(), self.lbx.data_ptr(),
                  self.ubx.data_ptr(), float(factor), float(constr_viol_tol),
                  self._s())
        self._relaxed = True
        self._host_bounds.pop("lbx", None)
        self._host_bounds.pop("ubx", None)

    # -- slacks (interior_point_optimizer.h:462-494) ----------------------
    def set_slack_mapping(self, slack_indices, constr_indices):
        si = np.ascontiguousarray(slack_indices, dtype=np.int32)
        ci = np.ascontiguousarray(constr_indices, dtype=np.int32)
        if si.shape != ci.shape:
            raise ValueError("slack and constraint index arrays differ in length")
        t = lambda a: torch.from_numpy(a).to(self.device)
        self._sidx, self._scidx = t(si), t(ci)
        self._nslack = len(si)

    def has_slacks(self):
        return self._nslack > 0

    def get_num_slacks(self):
        return self._nslack

    def initialize_slacks(self, grad, vars):
        """Slacks to the constraint bodies: s_k = (c_k(x) - s_k) + s_k from
        the gradient's constraint rows (evaluated at the current point)."""
        if self._nslack == 0:
            return
        _lib.call("ab_ipm_initialize_slacks", self._nslack, self._sidx.data_ptr(),
                  self._scidx.data_ptr(), _dev(grad).data_ptr(),
                  _dev(vars).data_ptr(), self._s())

    # -- NLP scaling (interior_point_optimizer.h:502-598) ------------------
    def compute_nlp_scaling(self, x, grad, max_gradient=100.0, min_value=1e-8):
        """Objective scale min(1, max_gradient / ||grad_f||_inf) and, per
        constraint row j of the KKT at x, dc_j = min(1, max_gradient /
        ||J_j||_inf) (both floored at min_value); the constraint targets
        are scaled by dc."""
        out = torch.zeros(1, dtype=torch.float64, device=self.device)
        _lib.call("ab_vec_absmax_gather", self.np_, self.pidx.data_ptr(),
                  _dev(grad).data_ptr(), out.data_ptr(), self._s())
        gmax = float(out.item())
        scale = max_gradient / gmax if gmax > max_gradient else 1.0
        self._obj_scale = max(scale, min_value)
        if self.problem is None:
            raise RuntimeError("compute_nlp_scaling needs the problem object "
                               "(create_matrix / hessian)")
        hess = self.problem.create_matrix()
        self.problem.hessian(1.0, x, hess)
        self._dc = torch.zeros(self.nc_, dtype=torch.float64, device=self.device)
        self._scale = torch.ones(self.n, dtype=torch.float64, device=self.device)
        _lib.call("ab_ipm_constraint_scale", self.n, self.nc_, self.cidx.data_ptr(),
                  hess.d_rowp.data_ptr(), hess.vals.data_ptr(), float(max_gradient),
                  float(min_value), self._dc.data_ptr(), self.lbh.data_ptr(),
                  self._scale.data_ptr(), self._s())
        self._scaling = True

    def apply_gradient_scaling(self, grad):
        if self._scaling:
            _lib.call("ab_vec_scale_gather", self.nc_, self.cidx.data_ptr(),
                      self._dc.data_ptr(), _dev(grad).data_ptr(), 0, self._s())

    def apply_hessian_scaling(self, hess):
        """D H D with D = 1 on primals and dc on the constraint rows."""
        if self._scaling:
            _lib.call("ab_csr_scale_symmetric", hess.nrows, hess.d_rowp.data_ptr(),
                      hess.d_cols.data_ptr(), self._scale.data_ptr(),
                      hess.vals.data_ptr(), self._s())

    def scale_multipliers(self, x):
        if self._scaling:
            _lib.call("ab_vec_scale_gather", self.nc_, self.cidx.data_ptr(),
                      self._dc.data_ptr(), _dev(x).data_ptr(), 0, self._s())

    def unscale_multipliers(self, x):
        if self._scaling:
            _lib.call("ab_vec_scale_gather", self.nc_, self.cidx.data_ptr(),
                      self._dc.data_ptr(), _dev(x).data_ptr(), 1, self._s())

    def get_obj_scale(self):
        return self._obj_scale

    def has_scaling(self):
        return self._scaling

    # -- copies and debug hooks --------------------------------------------
    def copy_multipliers(self, d, s):
        """d[constraint rows] = s[constraint rows]."""
        _lib.call("ab_vec_copy_gather", self.nc_, self.cidx.data_ptr(),
                  _dev(s).data_ptr(), _dev(d).data_ptr(), self._s())

    def copy_design_vars(self, d, s):
        _lib.call("ab_vec_copy_gather", self.np_, self.pidx.data_ptr(),
                  _dev(s).data_ptr(), _dev(d).data_ptr(), self._s())

    def compute_dual_residual_vector(self, vars, grad, out):
        """out = grad - zl + zu on the primals, 0 on the multipliers."""
        _lib.call("ab_ipm_dual_residual_vector", self.n, self.np_,
                  self.pidx.data_ptr(), _dev(grad).data_ptr(), vars.zl.data_ptr(),
                  vars.zu.data_ptr(), _dev(out).data_ptr(), self._s())

    def check_update(self, mu, grad, vars, update, hess):
        """Debug hook; a no-op, as in the reference
        (interior_point_optimizer.h:451-457)."""
        return None

    def initialize_multipliers_and_slacks(self, mu, grad, vars, kappa1=1e-2,
                                          kappa2=1e-2):
        _lib.call("ab_ipm_initialize", ctypes.byref(self._p),
                  vars.x.data_ptr(), vars.zl.data_ptr(), vars.zu.data_ptr(),
                  vars.sl.data_ptr(), vars.su.data_ptr(), float(kappa1),
                  float(kappa2), self._s())

    def set_multipliers_value(self, v, x):
        _dev(x)[self.cidx.long()] = v

    def set_design_vars_value(self, v, x):
        _dev(x)[self.pidx.long()] = v

    # -- Newton system ---------------------------------------------------
    def compute_residual(self, mu, vars, grad, res):
        r = _dev(res)
        r.zero_()
        self._c("ab_ipm_residual", ctypes.byref(self._state(vars)), float(mu),
                _dev(grad).data_ptr(), r.data_ptr(), None, self._s())
        return float(torch.linalg.vector_norm(r).item())

    def compute_residual_and_infeasibility(self, mu, vars, grad, res):
        r = _dev(res)
        r.zero_()
        self._c("ab_ipm_residual", ctypes.byref(self._state(vars)), float(mu),
                _dev(grad).data_ptr(), r.data_ptr(), self._out.data_ptr(),
                self._s())
        o = self._out[:2].cpu().numpy()
        return float(o[0]), float(o[1])

    def compute_diagonal(self, vars, diag):
        self._c("ab_ipm_diagonal", ctypes.byref(self._state(vars)),
                _dev(diag).data_ptr(), self._s())

    def compute_update(self, mu, vars, px, upd):
        upd.x.copy_(_dev(px))
        self._c("ab_ipm_bound_dual_step", ctypes.byref(self._state(vars)),
                float(mu), _dev(px).data_ptr(), upd.zl.data_ptr(),
                upd.zu.data_ptr(), self._s())

    # -- step ------------------------------------------------------------
    def compute_max_step(self, tau, vars, upd):
        self._c("ab_ipm_max_step", ctypes.byref(self._state(vars)), float(tau),
                upd.x.data_ptr(), upd.zl.data_ptr(), upd.zu.data_ptr(),
                self._out.data_ptr(), self._iout.data_ptr(), self._s())
        o = self._out[:2].cpu().numpy()
        i = self._iout[:2].cpu().numpy()
        return float(o[0]), int(i[0]), float(o[1]), int(i[1])

    def apply_step_update(self, ax, az, vars, upd, tmp):
        self._c("ab_ipm_apply_step", ctypes.byref(self._state(vars)),
                float(ax), float(az), upd.x.data_ptr(), upd.zl.data_ptr(),
                upd.zu.data_ptr(), tmp.x.data_ptr(), tmp.zl.data_ptr(),
                tmp.zu.data_ptr(), tmp.sl.data_ptr(), tmp.su.data_ptr(),
                self._s())

    def reset_bound_multipliers(self, barrier_param, kappa_sigma, vars):
        self._c("ab_ipm_reset_bound_multipliers",
                ctypes.byref(self._state(vars)), float(barrier_param),
                float(kappa_sigma), vars.zl.data_ptr(), vars.zu.data_ptr(),
                self._s())

    def compute_affine_start_point(self, beta_min, vars, upd, dst):
        self._c("ab_ipm_affine_start_point", ctypes.byref(self._state(vars)),
                float(beta_min), upd.zl.data_ptr(), upd.zu.data_ptr(),
                dst.zl.data_ptr(), dst.zu.data_ptr(), self._s())

    # -- reductions ------------------------------------------------------
    def _reduce(self, vars, mu=0.0, grad=None):
        self._c("ab_ipm_reductions", ctypes.byref(self._state(vars)),
                float(mu), None if grad is None else _dev(grad).data_ptr(),
                self._out.data_ptr(), self._s())
        return self._out[:13].cpu().numpy()

    def compute_complementarity(self, vars):
        o = self._reduce(vars)
        avg = o[0] / o[1] if o[1] > 0 else 0.0
        gm = o[2] if np.isfinite(o[2]) else np.finfo(np.float64).max
        xi = max(0.0, min(1.0, gm / avg)) if avg > 0 else 1.0
        return float(avg), float(xi)

    def compute_complementarity_sq(self, vars):
        return float(self._reduce(vars, 0.0)[9])

    def compute_max_comp_deviation(self, vars, mu):
        return float(self._reduce(vars, mu)[8])

    def compute_kkt_error(self, vars, grad):
        o = self._reduce(vars, 0.0, grad)
        return float(o[10]), float(o[11]), float(o[12])

    def compute_kkt_error_mu(self, mu, vars, grad):
        o = self._reduce(vars, mu, grad)
        return float(o[3]), float(o[4]), float(o[5])

    def compute_constraint_violation_1norm(self, vars, grad):
        return float(self._reduce(vars, 0.0, grad)[7])

    def compute_barrier_log_sum(self, barrier_param, vars):
        return float(self._reduce(vars, barrier_param)[6])

    def compute_barrier_dphi_direct(self, barrier_param, vars, grad, px):
        self._c("ab_ipm_barrier_dphi", ctypes.byref(self._state(vars)),
                float(barrier_param), _dev(grad).data_ptr(),
                _dev(px).data_ptr(), self._out.data_ptr(), self._s())
        return float(self._out[0].item())

    def compute_barrier_dphi(self, barrier_param, vars, update, res, px, diag):
        self._c("ab_ipm_barrier_dphi_kkt", ctypes.byref(self._state(vars)),
                _dev(res).data_ptr(), _dev(px).data_ptr(),
                _dev(diag).data_ptr(), self._out.data_ptr(), self._s())
        return float(self._out[0].item())


class BatchedInteriorPointOptimizer(InteriorPointOptimizer):
    """InteriorPointOptimizer over independent instances stored one after
    another (`vinst[i]` = instance of entry i, non-decreasing).  Every
    kernel that takes the barrier parameter reads instance k's value from
    `mu` (a device array set with set_barrier_params); seg_reduce returns
    per-instance norms, step lengths and merit terms, and
    apply_step_seg / the *_seg refinement steps act per instance."""

    def __init__(self, mult, lower, upper, vinst, device=None):
        super().__init__(mult, lower, upper, device=device)
        vinst = np.ascontiguousarray(vinst, dtype=np.int32)
        if len(vinst) != self.n or np.any(np.diff(vinst) < 0):
            raise ValueError("vinst must be non-decreasing with one entry per row")
        self.ninst = int(vinst[-1]) + 1 if len(vinst) else 0
        pidx, cidx = self.pidx.cpu().numpy(), self.cidx.cpu().numpy()
        pinst, cinst = vinst[pidx], vinst[cidx]
        cnt = lambda a: np.concatenate([[0], np.cumsum(np.bincount(a, minlength=self.ninst))])
        poff, coff = cnt(pinst).astype(np.int32), cnt(cinst).astype(np.int32)
        self.np_each = np.diff(poff)
        self.nc_each = np.diff(coff)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.vinst, self.pinst = t(vinst), t(pinst)
        self.poff, self.coff = t(poff), t(coff)
        f64 = dict(dtype=torch.float64, device=self.device)
        self.mu = torch.zeros(self.ninst, **f64)
        self.mu0 = torch.zeros(self.ninst, **f64)
        self._seg = torch.zeros(self.ninst * 12, **f64)
        self._ir = torch.zeros(self.ninst * 2, **f64)
        self._p = self._mk(self.mu)
        self._pz = self._mk(self.mu0)

    def _mk(self, mu):
        p = _lib.IpmProblem(self.n, self.np_, self.nc_, self.pidx.data_ptr(),
                            self.cidx.data_ptr(), self.lbx.data_ptr(),
                            self.ubx.data_ptr(), self.lbh.data_ptr())
        p.mu_inst, p.pinst, p.vinst = mu.data_ptr(), self.pinst.data_ptr(), self.vinst.data_ptr()
        p.ninst, p.poff, p.coff = self.ninst, self.poff.data_ptr(), self.coff.data_ptr()
        return p

    def set_barrier_params(self, mu):
        self.mu.copy_(torch.as_tensor(np.asarray(mu, dtype=np.float64)))

    def residual(self, vars, grad, res):
        """compute_residual with each instance's barrier parameter (no
        norm, no synchronisation)."""
        r = _dev(res)
        r.zero_()
        self._c("ab_ipm_residual", ctypes.byref(self._state(vars)), 0.0,
                _dev(grad).data_ptr(), r.data_ptr(), None, self._s())

    def seg_reduce_device(self, vars, grad=None, upd=None, gf=None, tau=0.0,
                          zero_mu=False):
        """seg_reduce into the device array `_seg` ((ninst, 12) doubles),
        with no copy to the host."""
        p = self._pz if zero_mu else self._p
        ptr = lambda a: None if a is None else a.data_ptr()
        _lib.call("ab_ipm_seg_reduce", ctypes.byref(p),
                  ctypes.byref(self._state(vars)), float(tau),
                  ptr(None if grad is None else _dev(grad)),
                  ptr(None if upd is None else upd.x),
                  ptr(None if upd is None else upd.zl),
                  ptr(None if upd is None else upd.zu),
                  ptr(None if gf is None else _dev(gf)),
                  self._seg.data_ptr(), self._s())
        return self._seg

    def seg_reduce(self, vars, grad=None, upd=None, gf=None, tau=0.0,
                   zero_mu=False):
        """Per-instance quantities as a (ninst, 12) host array (see
        ab_ipm_seg_reduce): 0 dual, 1 primal, 2 comp inf-norms, 3 constraint
        violation 1-norm, 4 barrier log-sum, 5/6 primal/dual step,
        7 barrier directional derivative, 8 max |lam + dlam|, 9/10 largest
        and smallest gap product."""
        self.seg_reduce_device(vars, grad, upd, gf, tau, zero_mu)
        return self._seg.view(self.ninst, 12).cpu().numpy()

    def apply_step_seg(self, ax, az, vars, upd, tmp):
        """tmp = vars + (ax[k], az[k]) * upd per instance; ax, az device."""
        self._c("ab_ipm_apply_step_seg", ctypes.byref(self._state(vars)),
                ax.data_ptr(), az.data_ptr(), upd.x.data_ptr(),
                upd.zl.data_ptr(), upd.zu.data_ptr(), tmp.x.data_ptr(),
                tmp.zl.data_ptr(), tmp.zu.data_ptr(), tmp.sl.data_ptr(),
                tmp.su.data_ptr(), self._s())
