"""Continuous-batching interior-point engine for many independent problems.

`BatchEngine` runs the interior-point loop of `ipm_driver.solve` (monotone
barrier update, inertia correction, 8-block refinement, fraction to the
boundary, l1-merit line search, bound-multiplier reset) on a changing set
of cart-pole instances: every phase of an iteration is one launch over all
instances -- the block-diagonal multifrontal LDL^T of
`linalg.BatchedSparseLDL`, the per-instance IPM kernels of
`ipm.BatchedInteriorPointOptimizer` -- while every decision (barrier
parameter, inertia correction, refinement stopping, step lengths, line
search) is taken per instance, on the device: the decision kernels of
csrc/batch_ctrl.cu (ab_bctl_*) read the per-instance reductions, inertia
and objectives where the other kernels left them, so an iteration moves no
per-instance array to the host; the host reads one flags word at the end of
each loop (inertia correction, refinement, line search) and the retired
instances' results.  Because no computation mixes instances, an instance's
iterates do not depend on which other instances share its batch.

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
from ._lib import (BCTL_IC_PENDING, BCTL_LIVE, BCTL_MISMATCH, BCTL_NFLAGS,
                   BCTL_REFINING, BCTL_RETIRED, BCTL_SEARCHING, BCTL_STALLED,
                   BctlOpts, BctlStruct)
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
        self.fallbacks = 0          # FP64 re-solves after a stalled refinement
        self.inertia_fallbacks = 0  # FP64 refactorizations on an FP32 inertia mismatch
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
        mu, nu = self.cd["mu"].cpu().numpy(), self.cd["nu"].cpu().numpy()
        dw_last = self.cd["dw_last"].cpu().numpy()
        n_ic = self.ci["n_ic"].cpu().numpy()
        for k, r in enumerate(self.insts):
            if r.done:
                continue
            a, b = int(B.var_off[k]), int(B.var_off[k + 1])
            p0, p1 = int(poff[k]), int(poff[k + 1])
            r.state = (st.x[a:b].clone(), st.zl[p0:p1].clone(),
                       st.zu[p0:p1].clone(), st.sl[p0:p1].clone(),
                       st.su[p0:p1].clone())
            r.mu, r.nu = float(mu[k]), float(nu[k])
            r.dw_last, r.n_ic = float(dw_last[k]), int(n_ic[k])

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
        opt.set_barrier_params(np.array([r.mu for r in self.insts]))
        # the per-instance decision state on the device (ab_bctl); its mu is
        # the barrier array the batched IPM kernels read
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
        self.cd = {k: torch.zeros(K, **f64) for k in BctlStruct.DOUBLES}
        self.cd["mu"] = opt.mu
        self.cd["nu"] = t([r.nu for r in self.insts], torch.float64)
        self.cd["dw_last"] = t([r.dw_last for r in self.insts], torch.float64)
        i32 = dict(dtype=torch.int32, device=dev)
        self.ci = {k: torch.zeros(K, **i32) for k in BctlStruct.INTS}
        self.ci["live"].fill_(1)
        self.ci["its"] = t([r.it for r in self.insts], torch.int32)
        self.ci["n_ic"] = t([r.n_ic for r in self.insts], torch.int32)
        self.ci["np_each"] = t(opt.np_each, torch.int32)
        self.ci["nc_each"] = t(opt.nc_each, torch.int32)
        self.ci["n_each"] = t(self.ldl.n_each, torch.int32)
        self.flags_d = torch.zeros(BCTL_NFLAGS, **i32)
        self.flags_h = torch.zeros(BCTL_NFLAGS, dtype=torch.int32).pin_memory()
        self.ctl = BctlStruct(K, *([self.cd[k].data_ptr() for k in BctlStruct.DOUBLES]
                                   + [self.ci[k].data_ptr() for k in BctlStruct.INTS]
                                   + [self.flags_d.data_ptr()]))
        o = self.o
        self.copts = BctlOpts(*([float(o[k]) for k in BctlOpts.NAMES]
                                + [int(o["max_iter"])]))
        self.obj_t = torch.zeros(K, **f64)
        self.vinst32 = opt.vinst
        self.pinst32 = opt.pinst
        self.stream = _stream_ptr(dev)
        self._built = True

    # -- helpers -----------------------------------------------------------
    def _objective(self, v, out=None):
        out = self.obj if out is None else out
        self.dm.objective(v.x, out)
        return out

    def _ctl(self, name, *args):
        _lib.call("ab_bctl_" + name, ctypes.byref(self.ctl), *args, self.stream)

    def _flags(self):
        """The decision flags (one small copy and a stream synchronisation)."""
        self.flags_h.copy_(self.flags_d, non_blocking=True)
        torch.cuda.current_stream(self.dev).synchronize()
        return self.flags_h.tolist()

    def _direction(self, st, steps):
        """px = K^-1 res with per-instance 8-block refinement; the stopping
        rule runs on the device (ab_bctl_refine_step), the host only learns
        whether any instance still refines."""
        opt = self.opt
        P = ctypes.byref(opt._p)
        opt.residual(st, self.g, self.res)
        self.px.copy_(self.res)
        self.ldl.solve_device(self.px)
        if not steps:
            return
        S = ctypes.byref(opt._state(st))
        _lib.call("ab_ipm_refine_init_seg", P, S, self.g.data_ptr(),
                  self.res.data_ptr(), self.px.data_ptr(), self.izl.data_ptr(),
                  self.izu.data_ptr(), self.seg.data_ptr(), self.stream)
        self._ctl("refine_init", self.seg.data_ptr())
        for step in range(steps + 1):
            self.H.mult(self.px, self.kpx)
            _lib.call("ab_ipm_refine_residual_seg", P, S, self.g.data_ptr(),
                      self.res.data_ptr(), self.kpx.data_ptr(), self.px.data_ptr(),
                      self.izl.data_ptr(), self.izu.data_ptr(), self.ecnd.data_ptr(),
                      self.ezl.data_ptr(), self.ezu.data_ptr(), self.seg.data_ptr(),
                      self.stream)
            self._ctl("clear_flags")
            self._ctl("refine_step", self.seg.data_ptr(), step)
            # at step 0 every live instance refines (the rule stops from
            # step 1), so only later steps need the flags
            if step >= 1 and not self._flags()[BCTL_REFINING]:
                break
            self.corr.copy_(self.ecnd)
            self.ldl.solve_device(self.corr)
            _lib.call("ab_ipm_refine_update_seg", P, S, self.ci["on"].data_ptr(),
                      self.corr.data_ptr(), self.ezl.data_ptr(), self.ezu.data_ptr(),
                      self.px.data_ptr(), self.izl.data_ptr(), self.izu.data_ptr(),
                      self.stream)

    def _factorize(self, force_fp64=False):
        """Inertia-corrected factorization of every live instance's KKT
        (Algorithm IC on the device).  With FP32 fronts, an attempt whose
        inertia differs from the wanted one for any pending instance is
        factored again in FP64 and the correction decides on the FP64
        inertia (the mismatch may be an FP32 artefact); force_fp64 runs the
        whole loop in FP64."""
        dm, H, ldl, st = self.dm, self.H, self.ldl, self.st
        copts = ctypes.byref(self.copts)
        mixed = self.precision == "fp32"
        if mixed and force_fp64:
            ldl.set_precision("fp64")
        self._ctl("ic_begin")
        for attempt in range(41):
            self._ctl("shift_diag", self.n, self.vinst32.data_ptr(),
                      self.primal.data_ptr(), self.diag.data_ptr(), self.dtot.data_ptr())
            dm.hessian(st.x, 1.0, H.vals)
            H.add_diagonal(self.dtot)
            ldl.factor(H.vals)
            if mixed and not force_fp64:
                self._ctl("clear_flags")
                self._ctl("ic_check", ldl.inertia_device())
                if self._flags()[BCTL_MISMATCH]:
                    self.inertia_fallbacks += 1
                    ldl.set_precision("fp64")
                    ldl.factor(H.vals)
                    ldl.set_precision("fp32")
            self._ctl("clear_flags")
            self._ctl("ic_step", copts, ldl.inertia_device())
            if not self._flags()[BCTL_IC_PENDING]:
                break
        self._ctl("ic_end")
        if mixed and force_fp64:
            # the factor stays FP64 for this iteration's solves
            ldl.set_precision("fp32")

    def _retire_marked(self):
        """Results of the instances ab_bctl_converge_barrier retired."""
        retire = self.ci["retire"].cpu().numpy()
        e0 = self.cd["e0"].cpu().numpy()
        n_ic = self.ci["n_ic"].cpu().numpy()
        objv = self._objective(self.st).cpu().numpy()
        B = self.B
        out = []
        for k in np.nonzero(retire)[0]:
            r = self.insts[k]
            a, b = int(B.var_off[k]), int(B.var_off[k + 1])
            r.done = True
            r.n_ic = int(n_ic[k])
            r.result = dict(id=r.id, converged=bool(retire[k] == 1), iterations=int(r.it),
                            objective=float(objv[k]), kkt_error=float(e0[k]),
                            inertia_corrections=int(n_ic[k]),
                            x=self.st.x[a:b].cpu().numpy(),
                            t_done=time.perf_counter())
            out.append(r.result)
        return out

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
        copts = ctypes.byref(self.copts)
        # convergence test (E_0 <= tol) or iteration limit, then the
        # monotone barrier update, per instance on the device
        dm.gradient(st.x, 1.0, g)
        opt.seg_reduce_device(st, grad=g)
        self._ctl("clear_flags")
        self._ctl("converge_barrier", copts, opt._seg.data_ptr())
        f = self._flags()
        finished = self._retire_marked() if f[BCTL_RETIRED] else []
        if not f[BCTL_LIVE]:
            return finished
        # inertia-corrected factorization
        opt.compute_diagonal(st, diag)
        self._factorize()
        # Newton direction; a stalled refinement on FP32 fronts is redone
        # after the whole inertia correction in FP64 (the FP32 factor's
        # accepted inertia may not be the FP64 factor's)
        from .ipm_driver import DeviceBackend
        steps = o["refine_steps"]
        if self.precision == "fp32":
            steps = max(steps, DeviceBackend.mixed_refine_steps)
        self._direction(st, steps)
        if self.precision == "fp32":
            self._ctl("clear_flags")
            self._ctl("refine_stalled")
            if self._flags()[BCTL_STALLED]:
                self.fallbacks += 1
                self._factorize(force_fp64=True)
                self._direction(st, steps)
        opt.compute_update(0.0, st, self.px, upd)
        # instances that have retired take no step
        self._ctl("mask_update", n, opt.np_, self.vinst32.data_ptr(),
                  self.pinst32.data_ptr(), upd.x.data_ptr(), upd.zl.data_ptr(),
                  upd.zu.data_ptr())
        # fraction to the boundary, merit, line search
        self.xtmp.copy_(st.x)
        self.xtmp[self.mult_idx] = 0.0
        dm.gradient(self.xtmp, 1.0, self.gf)
        opt.seg_reduce_device(st, grad=g, upd=upd, gf=self.gf, tau=-o["tau_min"])
        self._ctl("ls_begin", opt._seg.data_ptr(), self._objective(st).data_ptr())
        trial.copy(st)
        alpha, az = self.cd["alpha"], self.cd["az"]
        for ls in range(o["max_ls"]):
            opt.apply_step_seg(alpha, az, st, upd, trial)
            dm.gradient(trial.x, 1.0, self.gt)
            opt.seg_reduce_device(trial, grad=self.gt)
            self._objective(trial, self.obj_t)
            self._ctl("clear_flags")
            self._ctl("ls_test", copts, opt._seg.data_ptr(), self.obj_t.data_ptr())
            if not self._flags()[BCTL_SEARCHING]:
                break
        self.st, self.trial = trial, st
        opt.reset_bound_multipliers(0.0, o["kappa_sigma"], self.st)
        self._ctl("end")
        for r in self.insts:
            if not r.done:
                r.it += 1
        return finished
