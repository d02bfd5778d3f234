"""B200Solver (amigo LinearSolver contract) on the GPU: factor with the
device-assembled KKT, inertia, solve, and the device iterative refinement
on the 8-block system against oracle/ir_oracle.py (pinned to the
reference's own function).  Tolerance: refined directions agree to 1e-9
relative; the refined 8-block residual ratio is below 1e-10."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from amigo_b200.ipm import InteriorPointOptimizer
from amigo_b200.linalg import Vector
from amigo_b200.problems.simp2d import Simp2D
from amigo_b200.solver import B200Solver, Simp2DProblem
from oracle import ir_oracle

pytestmark = pytest.mark.gpu


def setup(nx=24, ny=12, seed=0):
    m = Simp2D(nx, ny, seed=seed)
    prob = Simp2DProblem(m, "cuda:0")
    solver = B200Solver(prob)
    opt = InteriorPointOptimizer(m.mult, m.lower, m.upper, device="cuda:0")
    opt.relax_bounds()
    x = torch.from_numpy(m.initial_point()).cuda()
    r = np.random.RandomState(seed)
    x[m.lam0:] = torch.from_numpy(0.1 * r.randn(m.n - m.lam0)).cuda()
    v = opt.create_opt_vector(x)
    opt.initialize_multipliers_and_slacks(0.1, None, v)
    return m, prob, solver, opt, v


def test_factor_solve_refine():
    m, prob, solver, opt, v = setup()
    n = m.n
    mu = 0.1
    grad = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    prob.gradient(1.0, v.x, grad)
    diag = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    opt.compute_diagonal(v, diag)
    primal = torch.from_numpy(~m.mult).cuda()
    diag.add_(primal, alpha=1e-4)
    diag.sub_((~primal).double(), alpha=1e-8)
    solver.factor(1.0, v.x, diag)
    npos, nneg = solver.get_inertia()
    assert npos + nneg == n
    res = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    opt.compute_residual(mu, v, grad, res)
    rhs_saved = res.clone()
    px = torch.zeros_like(res)
    solver.solve(res, px)
    px0 = px.clone()
    lbx = opt.lbx.cpu().numpy()
    ubx = opt.ubx.cpu().numpy()
    steps, ratio = solver.iterative_refinement(
        mu, m.mult, rhs_saved, v, grad, lbx, ubx, px, None, None, max_steps=10)
    assert ratio is not None and steps >= 1
    # oracle: same system, host CSR, splu correction solves
    K = sp.csr_matrix((solver.hess.vals.cpu().numpy(), m.cols, m.rowp),
                      shape=(n, n))
    lu = spla.splu(K.tocsc())
    want, dzl, dzu, osteps, oratio = ir_oracle.iterative_refinement(
        K, lu.solve, mu, m.mult, rhs_saved.cpu().numpy(),
        grad.cpu().numpy(), v.zl.cpu().numpy(), v.zu.cpu().numpy(),
        v.sl.cpu().numpy(), v.su.cpu().numpy(), lbx, ubx, px0.cpu().numpy())
    got = px.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-9 * max(1.0, np.abs(want).max())
    assert abs(steps - osteps) <= 1
    # the unrefined solve already solves the condensed system
    r = K @ px0.cpu().numpy() - rhs_saved.cpu().numpy()
    assert np.abs(r).max() <= 1e-10 * (abs(K).sum(axis=1).max() *
                                       np.abs(px0.cpu().numpy()).max())


def test_vector_interface():
    m, prob, solver, opt, v = setup(8, 4)
    n = m.n
    diag = torch.ones(n, dtype=torch.float64, device="cuda:0")
    solver.factor(1.0, v.x, diag)
    bx = Vector(n, device="cuda:0")
    bx.get_array()[:] = np.random.RandomState(1).randn(n)
    bx.copy_host_to_device()
    px = Vector(n, device="cuda:0")
    solver.solve(bx, px)
    px.copy_device_to_host()
    K = sp.csr_matrix((solver.hess.vals.cpu().numpy(), m.cols, m.rowp),
                      shape=(n, n))
    assert np.abs(K @ px.get_array() - bx.get_array()).max() <= 1e-9
    d = solver.assemble_hessian(1.0, v.x)
    assert d.shape == (n,)
