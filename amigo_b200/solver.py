"""B200Solver: amigo's LinearSolver plug-in contract on the GPU.

amigo's Optimizer accepts any object with the LinearSolver contract
(amigo/algorithm/solvers/linear_solver.py:6-107): factor(alpha, x, diag,
post_hessian=None), solve(bx, px), supports_inertia, get_inertia(), and the
DirectSparseSolver extras the inertia corrector and the Newton step call:
assemble_hessian(alpha, x), add_diagonal_and_factor(diag), the `hess`
attribute and iterative_refinement(...).  B200Solver keeps all of it on the
device: the KKT values are assembled by the problem's device kernels, the
factorization, inertia and solves are libamigo_b200.so's multifrontal LDL^T,
and iterative refinement on the unreduced 8-block system runs as device
kernels with one host read of the stopping ratio per step (the reference's
loop is host-driven in the same way).

`problem` supplies create_matrix() -> CSRMat, hessian(alpha, x, hess) and
add_diagonal(diag, hess) like amigo's OptimizationProblem
(include/optimization_problem.h:596-682, 801-818).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .linalg import OrderingType, SparseLDL, Vector, _stream_ptr


def _dev(v):
    return v.dev if isinstance(v, Vector) else v


class B200Solver:
    supports_inertia = True

    def __init__(self, problem, ustab=0.01, pivot_tol=1e-14, delay_growth=2.0,
                 order=OrderingType.DEFAULT, precision="fp64"):
        """precision "fp32" factors with FP32 fronts (mixed precision); the
        caller's iterative refinement against the FP64 KKT recovers FP64
        accuracy (see ipm_driver.DeviceBackend for the FP64 fallback)."""
        self.problem = problem
        self.hess = problem.create_matrix()
        (self.nrows, self.ncols, self.nnz, self.rowp,
         self.cols) = self.hess.get_nonzero_structure()
        self._diag_indices = self.hess.diag
        self.device = self.hess.device
        self.ldl = SparseLDL(self.hess, ustab=ustab, pivot_tol=pivot_tol,
                             delay_growth=delay_growth, order=order,
                             precision=precision)
        self.precision = precision
        self._ir = None
        self.last_refinement = None

    # -- factorization ----------------------------------------------------
    def factor(self, alpha, x, diag, post_hessian=None):
        self.problem.hessian(alpha, x, self.hess)
        if post_hessian is not None:
            post_hessian(self.hess)
        self.problem.add_diagonal(diag, self.hess)
        self.ldl.factor()

    def set_precision(self, precision):
        self.ldl.set_precision(precision)
        self.precision = precision

    def add_diagonal_and_factor(self, diag):
        self.problem.add_diagonal(diag, self.hess)
        self.ldl.factor()

    def assemble_hessian(self, alpha, x):
        """Assemble the Hessian and return its diagonal entries (host)."""
        self.problem.hessian(alpha, x, self.hess)
        return self.hess.vals[self.hess.d_diag.long()].cpu().numpy()

    def get_hessian_diagonal(self, alpha, x):
        return self.assemble_hessian(alpha, x)

    def get_inertia(self):
        return self.ldl.get_inertia()

    # -- solves -----------------------------------------------------------
    def solve(self, bx, px):
        p = _dev(px)
        p.copy_(_dev(bx))
        self.ldl.solve_device(p)

    # -- refinement -------------------------------------------------------
    def _ir_setup(self, mult_ind, lbx, ubx):
        # device copies of the index sets and bounds, rebuilt when any of
        # them changes (compared by value)
        mult_ind = np.asarray(mult_ind, dtype=bool)
        lbx = np.asarray(lbx, dtype=np.float64)
        ubx = np.asarray(ubx, dtype=np.float64)
        ir = self._ir
        if ir is not None and np.array_equal(ir["key"][0], mult_ind) and \
                np.array_equal(ir["key"][1], lbx) and np.array_equal(ir["key"][2], ubx):
            return ir
        key = (mult_ind.copy(), lbx.copy(), ubx.copy())
        pidx = np.nonzero(~mult_ind)[0].astype(np.int32)
        cidx = np.nonzero(mult_ind)[0].astype(np.int32)
        t = lambda a: torch.from_numpy(np.array(a, copy=True)).to(self.device)
        ir = dict(key=key, pidx=t(pidx), cidx=t(cidx),
                  lbx=t(np.asarray(lbx, dtype=np.float64)),
                  ubx=t(np.asarray(ubx, dtype=np.float64)),
                  lbh=t(np.zeros(len(cidx))))
        f64 = dict(dtype=torch.float64, device=self.device)
        n, npr = self.nrows, len(pidx)
        ir.update(kpx=torch.zeros(n, **f64), ecnd=torch.zeros(n, **f64),
                  corr=torch.zeros(n, **f64), dzl=torch.zeros(npr, **f64),
                  dzu=torch.zeros(npr, **f64), ezl=torch.zeros(npr, **f64),
                  ezu=torch.zeros(npr, **f64), out=torch.zeros(4, **f64))
        ir["p"] = _lib.IpmProblem(n, npr, len(cidx), ir["pidx"].data_ptr(),
                                  ir["cidx"].data_ptr(), ir["lbx"].data_ptr(),
                                  ir["ubx"].data_ptr(), ir["lbh"].data_ptr())
        self._ir = ir
        return ir

    def iterative_refinement(self, mu, mult_ind, rhs_saved, vars_, grad, lbx,
                             ubx, px, res, corr, max_steps=10):
        """Refine px on the unreduced 8-block system; same stopping rules as
        the reference (ratio < 1e-10 after >= 1 step, or improvement by less
        than a factor 0.999999999; at most max_steps)."""
        ir = self._ir_setup(mult_ind, lbx, ubx)
        s = _stream_ptr(self.device)
        st = _lib.IpmState(0, vars_.zl.data_ptr(), vars_.zu.data_ptr(),
                           vars_.sl.data_ptr(), vars_.su.data_ptr())
        P = ctypes.byref(ir["p"])
        pxd, g = _dev(px), _dev(grad)
        rhs = _dev(rhs_saved)
        if not torch.is_tensor(rhs):
            rhs = torch.as_tensor(np.asarray(rhs, dtype=np.float64), device=self.device)
        out = ir["out"]
        _lib.call("ab_ipm_refine_init", P, ctypes.byref(st), float(mu),
                  g.data_ptr(), rhs.data_ptr(), pxd.data_ptr(),
                  ir["dzl"].data_ptr(), ir["dzu"].data_ptr(), out.data_ptr(), s)
        nrm_rhs = float(out[0].item())
        ratio_old = 1e30
        steps = 0
        ratio = None
        for step in range(max_steps):
            self.hess.mult(pxd, ir["kpx"])
            _lib.call("ab_ipm_refine_residual", P, ctypes.byref(st), float(mu),
                      g.data_ptr(), rhs.data_ptr(), ir["kpx"].data_ptr(),
                      pxd.data_ptr(), ir["dzl"].data_ptr(), ir["dzu"].data_ptr(),
                      ir["ecnd"].data_ptr(), ir["ezl"].data_ptr(),
                      ir["ezu"].data_ptr(), out.data_ptr(), s)
            nres, nsol = out[:2].tolist()
            ratio = nres / (min(nsol, 1e6 * nrm_rhs) + nrm_rhs)
            if ratio < 1e-10 and step >= 1:
                break
            if step >= 1 and ratio > 0.999999999 * ratio_old:
                break
            ratio_old = ratio
            ir["corr"].copy_(ir["ecnd"])
            self.ldl.solve_device(ir["corr"])
            _lib.call("ab_ipm_refine_update", P, ctypes.byref(st),
                      ir["corr"].data_ptr(), ir["ezl"].data_ptr(),
                      ir["ezu"].data_ptr(), pxd.data_ptr(),
                      ir["dzl"].data_ptr(), ir["dzu"].data_ptr(), s)
            steps += 1
        self.last_refinement = (steps, ratio)
        return steps, ratio


class Simp2DProblem:
    """Device KKT problem for the 2D SIMP model (problems/simp2d.py):
    the `problem` B200Solver expects."""

    def __init__(self, model, device="cuda"):
        from .linalg import CSRMat
        self.model = model
        self.device = torch.device(device)
        self.dm = model.device_model(self.device)
        self._csr = CSRMat
        self.n = model.n

    def get_multiplier_indicator(self):
        return self.model.mult

    def create_matrix(self):
        m = self.model
        return self._csr(m.n, m.n, m.rowp, m.cols, device=self.device)

    def hessian(self, alpha, x, hess):
        self.dm.hessian(_dev(x), alpha, hess.vals)

    def gradient(self, alpha, x, g):
        self.dm.gradient(_dev(x), alpha, _dev(g))

    def add_diagonal(self, diag, hess):
        hess.add_diagonal(diag)
