"""Host numeric core for amigo_b200.ipm_driver (test infrastructure and the
CPU-baseline leg only).

Every numeric step the driver asks for is done by the reference's own code
where the reference has it: the KKT factorization, inertia and solve by its
SparseLDL (oracle/_ref, include/sparse_ldl.h), the IPM vector functions by
its include/interior_point_backend.h (oracle/_ref), the iterative
refinement by the restatement oracle/ir_oracle.py (pinned to
amigo/algorithm/solvers/linear_solver.py), and the cart-pole derivatives
by oracle/cartpole_oracle.py.  Running the same driver over this backend
and over amigo_b200.ipm_driver.DeviceBackend compares iteration counts and
optima of the two numeric cores.
"""
import numpy as np
import scipy.sparse as sp

from oracle import cartpole_oracle, ir_oracle, ref


class HostState:
    def __init__(self, x, zl, zu, sl, su):
        self.x, self.zl, self.zu, self.sl, self.su = x, zl, zu, sl, su

    def tup(self):
        return (self.x, self.zl, self.zu, self.sl, self.su)

    def copy(self):
        return HostState(*[a.copy() for a in self.tup()])


class HostBackend:
    def __init__(self, model, derivs=cartpole_oracle):
        self.m = model
        self.D = derivs
        mult = model.mult
        self.n = model.n
        self.pidx = np.nonzero(~mult)[0].astype(np.int32)
        self.cidx = np.nonzero(mult)[0].astype(np.int32)
        self.np, self.nc = len(self.pidx), len(self.cidx)
        lbx = model.lower[self.pidx].copy()
        ubx = model.upper[self.pidx].copy()
        # relax_bounds (interior_point_backend.h:126-146)
        for arr, sgn in ((lbx, -1.0), (ubx, 1.0)):
            fin = np.isfinite(arr)
            arr[fin] += sgn * np.minimum(1e-4, 1e-8 * np.maximum(1.0, np.abs(arr[fin])))
        self.lbx, self.ubx = lbx, ubx
        self.ipm = ref.RefIPM(self.pidx, self.cidx, lbx, ubx, model.lower[self.cidx])
        self.ldl = ref.RefSparseLDL(model.n, model.rowp, model.cols, order="AMD")
        self.primal = (~mult).astype(float)
        self.K = None

    def initial_state(self):
        x = self.m.x0.copy()
        lb, ub = self.lbx, self.ubx
        xp = x[self.pidx]
        hl, hu = np.isfinite(lb), np.isfinite(ub)
        both = hl & hu
        rng = np.where(both, ub - lb, 0.0)
        pl = np.minimum(1e-2 * np.maximum(1.0, np.abs(lb)), 1e-2 * rng)
        pu = np.minimum(1e-2 * np.maximum(1.0, np.abs(ub)), 1e-2 * rng)
        xp = np.where(both, np.maximum(np.minimum(xp, ub - pu), lb + pl), xp)
        onlyl = hl & ~hu
        onlyu = hu & ~hl
        with np.errstate(invalid="ignore"):
            xp = np.where(onlyl, np.maximum(xp, lb + 1e-2 * np.maximum(1.0, np.abs(lb))), xp)
            xp = np.where(onlyu, np.minimum(xp, ub - 1e-2 * np.maximum(1.0, np.abs(ub))), xp)
        x[self.pidx] = xp
        zl = np.where(hl, 1.0, 0.0)
        zu = np.where(hu, 1.0, 0.0)
        sl = np.where(hl, xp - lb, 1.0)
        su = np.where(hu, ub - xp, 1.0)
        return HostState(x, zl, zu, sl, su)

    def gradient(self, st):
        return self.D.gradient(self.m, st.x, 1.0)

    def objective_gradient(self, st):
        x = st.x.copy()
        x[self.cidx] = 0.0
        return self.D.gradient(self.m, x, 1.0)

    def objective(self, st):
        return self.D.objective(self.m, st.x)

    def kkt_error(self, mu, st, g):
        return self.ipm.compute_kkt_error(mu, st.tup(), g)

    def diagonal(self, st):
        return self.ipm.compute_diagonal(st.tup(), self.n)

    def factor(self, st, diag, dw, dc, force_fp64=False):
        vals = self.D.hessian_values(self.m, st.x, 1.0)
        vals[self.m.diag_pos] += diag + dw * self.primal - dc * (1.0 - self.primal)
        self.vals = vals
        self.ldl.factor(vals)
        return self.ldl.inertia()

    def residual(self, mu, st, g):
        return self.ipm.compute_residual(mu, st.tup(), g)

    def solve(self, res):
        return self.ldl.solve(res)

    def refine(self, mu, st, g, res, px, steps):
        K = sp.csr_matrix((self.vals, self.m.cols, self.m.rowp), shape=(self.n, self.n))
        out, *_ = ir_oracle.iterative_refinement(
            K, self.ldl.solve, mu, self.m.mult, res, g, st.zl, st.zu, st.sl,
            st.su, self.lbx, self.ubx, px, max_steps=steps + 1)
        px[:] = out
        return True

    def update(self, mu, st, px):
        dzl, dzu = self.ipm.compute_bound_dual_step(mu, st.tup(), px)
        return (px.copy(), dzl, dzu)

    def max_step(self, tau, st, upd):
        ax, xi, az, zi = self.ipm.compute_max_step(tau, st.tup(), *upd)
        return ax, az

    def apply_step(self, ax, az, st, upd):
        out = self.ipm.apply_step(ax, az, st.tup(), *upd)
        return HostState(*out)

    def max_abs_mult(self, st, px):
        lam = st.x[self.cidx] + px[self.cidx]
        return float(np.abs(lam).max()) if len(lam) else 0.0

    def cviol(self, st, g):
        return self.ipm.compute_constraint_violation_1norm(st.tup(), g)

    def barrier_log_sum(self, mu, st):
        return self.ipm.compute_barrier_log_sum(mu, st.tup())

    def dphi(self, mu, st, gf, px):
        return self.ipm.compute_barrier_dphi(mu, st.tup(), gf, px)

    def reset_bound_multipliers(self, mu, kappa, st):
        zl, zu = self.ipm.reset_bound_multipliers(mu, kappa, st.tup())
        st.zl[:], st.zu[:] = zl, zu

    def solution(self, st):
        return st.x.copy()
