"""Pin oracle/ir_oracle.py (CPU restatement of the 8-block iterative
refinement) against the reference's own DirectSparseSolver
.iterative_refinement (amigo/algorithm/solvers/linear_solver.py:109-264),
executed here from the reference sources.  CPU only; skipped where the
reference sources are not present."""
import importlib.util
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import ir_oracle

REF = os.path.join(os.environ.get("AMIGO_REF_ROOT", "/root/reference"),
                   "amigo", "algorithm", "solvers", "linear_solver.py")


class _Arr:
    def __init__(self, a):
        self.a = a

    def get_array(self):
        return self.a

    def copy_host_to_device(self):
        pass

    def copy_device_to_host(self):
        pass


class _Vars:
    def __init__(self, zl, zu, sl, su):
        self.zl, self.zu, self.sl, self.su = zl, zu, sl, su

    def get_zl(self):
        return self.zl

    def get_zu(self):
        return self.zu

    def get_sl(self):
        return self.sl

    def get_su(self):
        return self.su


def problem(seed, n_primal=300, n_con=120):
    r = np.random.RandomState(seed)
    n = n_primal + n_con
    mult = np.zeros(n, bool)
    mult[r.choice(n, n_con, replace=False)] = True
    lbx = np.where(r.rand(n_primal) < 0.7, -1.0, -np.inf)
    ubx = np.where(r.rand(n_primal) < 0.5, 2.0, np.inf)
    zl, zu = 0.1 + r.rand(n_primal), 0.1 + r.rand(n_primal)
    sl, su = 0.05 + r.rand(n_primal), 0.05 + r.rand(n_primal)
    A = sp.random(n, n, density=0.02, random_state=r)
    K = (A + A.T + sp.diags(4.0 + r.rand(n))).tocsr()
    K.sort_indices()
    g = r.randn(n)
    rhs = r.randn(n)
    return mult, lbx, ubx, zl, zu, sl, su, K, g, rhs


@pytest.mark.skipif(not os.path.exists(REF), reason="reference sources absent")
def test_ir_restatement_matches_reference():
    spec = importlib.util.spec_from_file_location("ref_linear_solver", REF)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    for seed in range(3):
        mult, lbx, ubx, zl, zu, sl, su, K, g, rhs = problem(seed)
        n = K.shape[0]
        lu = spla.splu(K.tocsc())
        # perturbed first solve so that refinement has work to do
        px0 = lu.solve(rhs) * (1 + 1e-6 * np.random.RandomState(seed).randn(n))

        class S(mod.DirectSparseSolver):
            def _do_factor(self):
                pass

            def factor(self, *a):
                pass

            def solve(self, bx, px):
                px.get_array()[:] = lu.solve(bx.get_array())

        s = S()
        s.hess = type("H", (), {"copy_data_device_to_host": lambda self: None,
                                "get_data": lambda self: K.data})()
        s.rowp, s.cols = K.indptr, K.indices
        px = _Arr(px0.copy())
        res, corr = _Arr(np.zeros(n)), _Arr(np.zeros(n))
        s.iterative_refinement(0.1, mult, rhs, _Vars(zl, zu, sl, su), _Arr(g),
                               lbx, ubx, px, res, corr, max_steps=10)
        got, *_ = ir_oracle.iterative_refinement(
            K, lu.solve, 0.1, mult, rhs, g, zl, zu, sl, su, lbx, ubx, px0,
            max_steps=10)
        np.testing.assert_array_equal(got, px.a)
