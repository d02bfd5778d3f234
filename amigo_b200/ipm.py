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


class InteriorPointOptimizer:
    """Device IPM vector operations over a fixed primal/multiplier split.

    InteriorPointOptimizer(mult_indicator, lower, upper, device=None)
    matches the reference constructor's effect
    (include/interior_point_optimizer.h:114-166): primal entries keep
    [lower, upper] as bounds, multiplier entries take lower as lbh.
    """

    def __init__(self, mult, lower, upper, device=None):
        self.device = _device(device)
        mult = np.asarray(mult).astype(bool)
        lower = np.asarray(lower, dtype=np.float64)
        upper = np.asarray(upper, dtype=np.float64)
        self.n = len(mult)
        pidx = np.nonzero(~mult)[0].astype(np.int32)
        cidx = np.nonzero(mult)[0].astype(np.int32)
        self.np_, self.nc_ = len(pidx), len(cidx)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.pidx, self.cidx = t(pidx), t(cidx)
        self.lbx, self.ubx = t(lower[pidx]), t(upper[pidx])
        self.lbh = t(lower[cidx])
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

    # -- setup -----------------------------------------------------------
    def relax_bounds(self, factor=1e-8, constr_viol_tol=1e-4):
        _lib.call("ab_ipm_relax_bounds", self.np_, self.lbx.data_ptr(),
                  self.ubx.data_ptr(), self.lbx.data_ptr(),
                  self.ubx.data_ptr(), float(factor), float(constr_viol_tol),
                  self._s())

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
        self._seg = torch.zeros(self.ninst * 10, **f64)
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

    def seg_reduce(self, vars, grad=None, upd=None, gf=None, tau=0.0,
                   zero_mu=False):
        """Per-instance quantities as a (ninst, 10) host array (see
        ab_ipm_seg_reduce): 0 dual, 1 primal, 2 comp inf-norms, 3 constraint
        violation 1-norm, 4 barrier log-sum, 5/6 primal/dual step,
        7 barrier directional derivative, 8 max |lam + dlam|."""
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
        return self._seg.view(self.ninst, 10).cpu().numpy()

    def apply_step_seg(self, ax, az, vars, upd, tmp):
        """tmp = vars + (ax[k], az[k]) * upd per instance; ax, az device."""
        self._c("ab_ipm_apply_step_seg", ctypes.byref(self._state(vars)),
                ax.data_ptr(), az.data_ptr(), upd.x.data_ptr(),
                upd.zl.data_ptr(), upd.zu.data_ptr(), tmp.x.data_ptr(),
                tmp.zl.data_ptr(), tmp.zu.data_ptr(), tmp.sl.data_ptr(),
                tmp.su.data_ptr(), self._s())
