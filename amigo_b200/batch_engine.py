"""Continuous-batching interior-point engine for many independent problems.

`BatchEngine` runs the interior-point loop of `ipm_driver.solve` (monotone
barrier update, inertia correction, 8-block refinement, fraction to the
boundary, l1-merit line search, bound-multiplier reset) on a changing set
of cart-pole instances: every phase of an iteration is one launch over all
instances -- the block-diagonal multifrontal LDL^T of
`linalg.BatchedSparseLDL`, the per-instance IPM kernels of
`ipm.BatchedInteriorPointOptimizer` -- while every decision (barrier
parameter, inertia correction, refinement stopping, step lengths, line
search) is taken per instance.  Because no computation mixes instances, an
instance's iterates do not depend on which other instances share its batch.

Instances are admitted (`admit`) and retired (converged or out of
iterations) at iteration boundaries.  Admission rebuilds the batch: the
symbolic analysis of each pattern is cached by the library, the surviving
instances' iterates are copied into the new layout, and new instances start
from their initial point.  `ipm_driver.solve_batch` is the engine with one
admission; `serve.py` drives it from a request stream.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from .linalg import OrderingType, _stream_ptr


class _Inst:
    __slots__ = ("id", "model", "it", "mu", "nu", "dw_last", "n_ic", "state",
                 "done", "result")

    def __init__(self, rid, model, mu0):
        self.id = rid
        self.model = model
        self.it = 0
        self.mu = mu0
        self.nu = 1.0
        self.dw_last = 0.0
        self.n_ic = 0
        self.state = None     # (x, zl, zu, sl, su) device copies between layouts
        self.done = False
        self.result = None


class BatchEngine:
    def __init__(self, device="cuda", options=None, precision="fp64"):
        from .ipm_driver import DEFAULTS
        self.o = dict(DEFAULTS)
        self.o.update(options or {})
        self.dev = torch.device(device)
        self.precision = precision
        self.insts = []        # current layout, in batch order
        self.waiting = []      # admitted, not yet in the layout
        self.fallbacks = 0
        self.rebuilds = 0
        self.rebuild_s = 0.0   # host + device time spent rebuilding layouts
        self._built = False

    # -- membership ------------------------------------------------------
    def admit(self, items):
        """items: iterable of (request id, problems.cartpole.CartPole)."""
        for rid, m in items:
            self.waiting.append(_Inst(rid, m, self.o["mu0"]))

    def live(self):
        return sum(1 for r in self.insts if not r.done) + len(self.waiting)

    def dead_fraction(self):
        """Share of the current layout that has retired (stepped with zero
        steps until the next rebuild)."""
        if not self.insts:
            return 0.0
        return sum(1 for r in self.insts if r.done) / len(self.insts)

    def _save_states(self):
        if not self._built:
            return
        st, B, poff = self.st, self.B, self.poff
        for k, r in enumerate(self.insts):
            if r.done:
                continue
            a, b = int(B.var_off[k]), int(B.var_off[k + 1])
            p0, p1 = int(poff[k]), int(poff[k + 1])
            r.state = (st.x[a:b].clone(), st.zl[p0:p1].clone(),
                       st.zu[p0:p1].clone(), st.sl[p0:p1].clone(),
                       st.su[p0:p1].clone())
            r.mu, r.nu = float(self.mu[k]), float(self.nu[k])
            r.dw_last, r.n_ic = float(self.dw_last[k]), int(self.n_ic[k])

    def _build(self):
        from .ipm import BatchedInteriorPointOptimizer
        from .linalg import BatchedSparseLDL, CSRMat
        from .problems.cartpole import CartPoleBatch
        t0 = time.perf_counter()
        try:
            self._build_layout(BatchedInteriorPointOptimizer, BatchedSparseLDL,
                               CSRMat, CartPoleBatch)
        finally:
            self.rebuild_s += time.perf_counter() - t0

    def _build_layout(self, BatchedInteriorPointOptimizer, BatchedSparseLDL,
                      CSRMat, CartPoleBatch):
        self._save_states()
        self.insts = [r for r in self.insts if not r.done] + self.waiting
        self.waiting = []
        self.rebuilds += 1
        if not self.insts:
            self._built = False
            return
        dev = self.dev
        B = CartPoleBatch([r.model for r in self.insts])
        self.B = B
        self.K, self.n = B.k, B.n
        self.dm = B.device_model(dev)
        self.H = CSRMat(B.n, B.n, B.rowp, B.cols, device=dev, diag_pos=B.diag_pos)
        self.ldl = BatchedSparseLDL(B.patterns(), order=OrderingType.AMD, device=dev)
        if self.precision == "fp32":
            self.ldl.set_precision("fp32")
        opt = BatchedInteriorPointOptimizer(B.mult, B.lower, B.upper, B.vinst,
                                            device=dev)
        opt.relax_bounds()
        self.opt = opt
        self.poff = opt.poff.cpu().numpy()
        f64 = dict(dtype=torch.float64, device=dev)
        n, K = self.n, self.K
        self.vinst = opt.vinst.long()
        self.pinst = opt.pinst.long()
        self.primal = torch.from_numpy(~B.mult).to(dev).double()
        self.mult_idx = opt.cidx.long()
        (self.g, self.gf, self.res, self.px, self.diag, self.dtot, self.xtmp,
         self.kpx, self.ecnd, self.corr, self.gt) = (torch.zeros(n, **f64)
                                                     for _ in range(11))
        (self.ezl, self.ezu, self.izl, self.izu) = (torch.zeros(opt.np_, **f64)
                                                    for _ in range(4))
        self.seg = torch.zeros(2 * K, **f64)
        self.act = torch.zeros(K, dtype=torch.int32, device=dev)
        self.obj = torch.zeros(K, **f64)
        self.upd = opt.create_opt_vector()
        self.trial = opt.create_opt_vector()
        st = opt.create_opt_vector(torch.from_numpy(np.ascontiguousarray(B.x0)).to(dev))
        opt.initialize_multipliers_and_slacks(0.1, None, st)
        for k, r in enumerate(self.insts):
            if r.state is None:
                continue
            a, b = int(B.var_off[k]), int(B.var_off[k + 1])
            p0, p1 = int(self.poff[k]), int(self.poff[k + 1])
            st.x[a:b].copy_(r.state[0])
            st.zl[p0:p1].copy_(r.state[1])
            st.zu[p0:p1].copy_(r.state[2])
            st.sl[p0:p1].copy_(r.state[3])
            st.su[p0:p1].copy_(r.state[4])
            r.state = None
        self.st = st
        self.mu = np.array([r.mu for r in self.insts])
        self.nu = np.array([r.nu for r in self.insts])
        self.dw_last = np.array([r.dw_last for r in self.insts])
        self.n_ic = np.array([r.n_ic for r in self.insts], np.int64)
        opt.set_barrier_params(self.mu)
        self.stream = _stream_ptr(dev)
        self._built = True

    # -- helpers -----------------------------------------------------------
    def _dev_vec(self, a, dtype=torch.float64):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).to(self.dev)

    def _objective(self, v):
        self.dm.objective(v.x, self.obj)
        return self.obj.cpu().numpy()

    def _direction(self, st, steps, live):
        """px = K^-1 res with per-instance 8-block refinement; returns each
        instance's last residual ratio."""
        opt, K = self.opt, self.K
        P = ctypes.byref(opt._p)
        opt.residual(st, self.g, self.res)
        self.px.copy_(self.res)
        self.ldl.solve_device(self.px)
        ratio = np.zeros(K)
        if not steps:
            return ratio
        S = ctypes.byref(opt._state(st))
        _lib.call("ab_ipm_refine_init_seg", P, S, self.g.data_ptr(),
                  self.res.data_ptr(), self.px.data_ptr(), self.izl.data_ptr(),
                  self.izu.data_ptr(), self.seg.data_ptr(), self.stream)
        nrm_rhs = self.seg[:K].cpu().numpy()
        ratio_old = np.full(K, 1e30)
        on = live.copy()
        for step in range(steps + 1):
            self.H.mult(self.px, self.kpx)
            _lib.call("ab_ipm_refine_residual_seg", P, S, self.g.data_ptr(),
                      self.res.data_ptr(), self.kpx.data_ptr(), self.px.data_ptr(),
                      self.izl.data_ptr(), self.izu.data_ptr(), self.ecnd.data_ptr(),
                      self.ezl.data_ptr(), self.ezu.data_ptr(), self.seg.data_ptr(),
                      self.stream)
            ns = self.seg.view(K, 2).cpu().numpy()
            r = ns[:, 0] / (np.minimum(ns[:, 1], 1e6 * nrm_rhs) + nrm_rhs)
            ratio = np.where(on, r, ratio)
            if step >= 1:
                on &= ~((r < 1e-10) | (r > 0.999999999 * ratio_old))
            if not on.any():
                break
            ratio_old = np.where(on, r, ratio_old)
            self.corr.copy_(self.ecnd)
            self.ldl.solve_device(self.corr)
            self.act.copy_(self._dev_vec(on.astype(np.int32), torch.int32))
            _lib.call("ab_ipm_refine_update_seg", P, S, self.act.data_ptr(),
                      self.corr.data_ptr(), self.ezl.data_ptr(), self.ezu.data_ptr(),
                      self.px.data_ptr(), self.izl.data_ptr(), self.izu.data_ptr(),
                      self.stream)
        return ratio

    def _retire(self, k, converged, kkt, objective):
        r = self.insts[k]
        B = self.B
        a, b = int(B.var_off[k]), int(B.var_off[k + 1])
        r.done = True
        r.result = dict(id=r.id, converged=bool(converged), iterations=int(r.it),
                        objective=float(objective), kkt_error=float(kkt),
                        inertia_corrections=int(self.n_ic[k]),
                        x=self.st.x[a:b].cpu().numpy(),
                        t_done=time.perf_counter())
        return r.result

    # -- one iteration -------------------------------------------------------
    def step(self, rebuild=None):
        """One interior-point iteration of every live instance; admits the
        waiting ones first when `rebuild` (default: whenever some wait).
        Returns the results of the instances retired at its start."""
        if rebuild is None:
            rebuild = bool(self.waiting)
        if rebuild or not self._built:
            self._build()
        if not self._built:
            return []
        o, K, n = self.o, self.K, self.n
        opt, dm, H, ldl = self.opt, self.dm, self.H, self.ldl
        st, upd, trial = self.st, self.upd, self.trial
        g, diag, dtot, primal = self.g, self.diag, self.dtot, self.primal
        mu, nu, dw_last, n_ic = self.mu, self.nu, self.dw_last, self.n_ic
        dev_vec = self._dev_vec
        live = np.array([not r.done for r in self.insts])
        its = np.array([r.it for r in self.insts])
        finished = []
        # convergence test (E_0 <= tol) or iteration limit, per instance
        dm.gradient(st.x, 1.0, g)
        q = opt.seg_reduce(st, grad=g, zero_mu=True)
        E0 = q[:, :3].max(axis=1)
        conv = live & (E0 <= o["tol"])
        out = live & ~conv & (its >= o["max_iter"])
        if conv.any() or out.any():
            objv = self._objective(st)
            for k in np.nonzero(conv | out)[0]:
                finished.append(self._retire(k, conv[k], E0[k], objv[k]))
        live &= ~(conv | out)
        if not live.any():
            return finished
        # monotone barrier update
        while True:
            q = opt.seg_reduce(st, grad=g)
            Emu = q[:, :3].max(axis=1)
            dec = live & (Emu <= o["kappa_eps"] * mu) & (mu > o["mu_min"])
            if not dec.any():
                break
            mu[dec] = np.maximum(o["mu_min"], np.minimum(o["kappa_mu"] * mu[dec],
                                                         mu[dec] ** o["theta_mu"]))
            opt.set_barrier_params(mu)
        # inertia-corrected factorization
        opt.compute_diagonal(st, diag)
        dw, dc = np.zeros(K), np.zeros(K)
        dwf, dcf = dw.copy(), dc.copy()     # values the factor was made with
        pending = live.copy()
        for attempt in range(41):
            dwv, dcv = dev_vec(dwf)[self.vinst], dev_vec(dcf)[self.vinst]
            torch.addcmul(diag, dwv, primal, out=dtot)
            dtot.sub_(dcv * (1.0 - primal))
            dm.hessian(st.x, 1.0, H.vals)
            H.add_diagonal(dtot)
            ldl.factor(H.vals)
            inertia = np.array(ldl.get_inertia())
            ok = (inertia[:, 0] == opt.np_each) & (inertia[:, 1] == opt.nc_each)
            bad = pending & ~ok
            if not bad.any():
                break
            n_ic[bad] += 1
            sing = bad & (inertia.sum(axis=1) < ldl.n_each) & (dc == 0.0)
            dc[sing] = o["dc"] * mu[sing] ** o["kappa_c"]
            first = bad & (dw == 0.0)
            dw[first] = np.where(dw_last[first] == 0.0, o["dw_first"],
                                 np.maximum(o["dw_min"], o["kw_minus"] * dw_last[first]))
            grow = bad & ~first
            dw[grow] *= np.where(dw_last[grow] == 0.0, o["kw_plus_first"], o["kw_plus"])
            pending = bad & (dw <= o["dw_max"])
            dwf[pending], dcf[pending] = dw[pending], dc[pending]
            if not pending.any():
                break
        self.dw_last = np.where(live & (dw > 0.0), dw, dw_last)
        # Newton direction; a stalled refinement on FP32 fronts is redone on
        # an FP64 refactorization of the same matrices
        from .ipm_driver import DeviceBackend
        steps = o["refine_steps"]
        if self.precision == "fp32":
            steps = max(steps, DeviceBackend.mixed_refine_steps)
        ratio = self._direction(st, steps, live)
        if self.precision == "fp32" and np.any(live & (ratio > 1e-10)):
            self.fallbacks += 1
            ldl.set_precision("fp64")
            dm.hessian(st.x, 1.0, H.vals)
            H.add_diagonal(dtot)
            ldl.factor(H.vals)
            self._direction(st, steps, live)
            ldl.set_precision("fp32")
        opt.compute_update(0.0, st, self.px, upd)
        # instances that have retired take no step
        lv = dev_vec(live, torch.bool)
        upd.x.copy_(torch.where(lv[self.vinst], upd.x, 0.0))
        upd.duals.view(2, -1).copy_(torch.where(lv[self.pinst], upd.duals.view(2, -1), 0.0))
        # fraction to the boundary, merit, line search
        self.xtmp.copy_(st.x)
        self.xtmp[self.mult_idx] = 0.0
        dm.gradient(self.xtmp, 1.0, self.gf)
        q = opt.seg_reduce(st, grad=g, upd=upd, gf=self.gf, tau=-o["tau_min"])
        ax, az = q[:, 5].copy(), q[:, 6].copy()
        self.nu = nu = np.where(live, np.maximum(nu, 1.1 * q[:, 8]), nu)
        theta0 = q[:, 3]
        phi0 = self._objective(st) + q[:, 4] + nu * theta0
        dphi = q[:, 7] - nu * theta0
        alpha = np.where(live, ax, 0.0)
        az_d = dev_vec(np.where(live, az, 0.0))
        search = live.copy()
        trial.copy(st)
        for ls in range(o["max_ls"]):
            opt.apply_step_seg(dev_vec(alpha), az_d, st, upd, trial)
            dm.gradient(trial.x, 1.0, self.gt)
            qt = opt.seg_reduce(trial, grad=self.gt)
            phi = self._objective(trial) + qt[:, 4] + nu * qt[:, 3]
            accept = (phi <= phi0 + o["armijo"] * alpha * dphi) | ~np.isfinite(dphi)
            search &= ~accept
            if not search.any():
                break
            alpha = np.where(search, 0.5 * alpha, alpha)
        self.st, self.trial = trial, st
        opt.reset_bound_multipliers(0.0, o["kappa_sigma"], self.st)
        for k in np.nonzero(live)[0]:
            self.insts[k].it += 1
        return finished
