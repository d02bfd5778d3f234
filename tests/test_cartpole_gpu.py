"""Cart-pole swing-up collocation model (N = 100 intervals) on the GPU: the
hyper-dual component kernels against finite differences of the numpy
Lagrangian (oracle/cartpole_oracle.py), and the KKT factorization at the
seeded initial point against the reference's own SparseLDL (identical
symbolic arrays and inertia, residual <= 1e-10)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from amigo_b200 import linalg
from amigo_b200.problems.cartpole import CartPole
from oracle import cartpole_oracle as O

pytestmark = pytest.mark.gpu


def grad_hess(m, x, alpha=1.0):
    dm = m.device_model("cuda:0")
    xd = torch.from_numpy(x).cuda()
    g = torch.zeros(m.n, dtype=torch.float64, device="cuda:0")
    dm.gradient(xd, alpha, g)
    v = torch.zeros(m.nnz, dtype=torch.float64, device="cuda:0")
    dm.hessian(xd, alpha, v)
    return g.cpu().numpy(), v.cpu().numpy(), dm


def test_derivatives_against_finite_differences():
    m = CartPole(N=7, seed=3)
    r = np.random.RandomState(0)
    x = m.x0.copy()
    x[m.d0:] = r.randn(m.n - m.d0)
    g, v, dm = grad_hess(m, x, 0.8)
    h = 1e-6
    for i in range(m.n):
        e = np.zeros(m.n)
        e[i] = h
        fd = (O.lagrangian(m, x + e, 0.8) - O.lagrangian(m, x - e, 0.8)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), i
    K = sp.csr_matrix((v, m.cols, m.rowp), shape=(m.n, m.n)).toarray()
    assert np.abs(K - K.T).max() <= 1e-12 * max(1.0, np.abs(K).max())
    for i in range(m.n):
        e = np.zeros(m.n)
        e[i] = h
        gp, _, _ = grad_hess(m, x + e, 0.8)
        gm, _, _ = grad_hess(m, x - e, 0.8)
        fd = (gp - gm) / (2 * h)
        assert np.abs(fd - K[:, i]).max() <= 1e-5 * max(1.0, np.abs(K[:, i]).max()), i


def test_constraint_rows_are_constraint_values():
    m = CartPole(N=20, seed=1)
    x = m.x0.copy()
    g, _, _ = grad_hess(m, x)
    c = O.constraints(m, x)
    np.testing.assert_allclose(g[m.d0:], c[m.d0:], rtol=1e-12, atol=1e-12)


def test_kkt_factor_matches_reference(oracle_ref):
    m = CartPole(N=100, seed=0)
    x = m.x0.copy()
    x[m.d0:] = 0.1
    g, v, dm = grad_hess(m, x)
    prim = ~m.mult
    v[m.diag_pos[prim]] += 1.0   # barrier-like diagonal on the primals
    v[m.diag_pos[~prim]] -= 1e-8
    R = oracle_ref.RefSparseLDL(m.n, m.rowp, m.cols, order="AMD")
    R.factor(v)
    want = R.symbolic()
    got = linalg.analyze(m.n, m.rowp, m.cols, linalg.OrderingType.AMD)
    for k in ("node_ptr", "node_to_var", "children_ptr", "children",
              "contrib_ptr", "contrib_rows", "invperm"):
        np.testing.assert_array_equal(got[k], want[k])
    mat = linalg.CSRMat(m.n, m.n, m.rowp, m.cols, v)
    ldl = linalg.SparseLDL(mat, order=linalg.OrderingType.AMD)
    ldl.factor()
    assert ldl.get_inertia() == R.inertia()
    K = sp.csr_matrix((v, m.cols, m.rowp), shape=(m.n, m.n))
    b = K @ np.random.RandomState(2).randn(m.n)
    xs = b.copy()
    ldl.solve(xs)
    res = np.abs(K @ xs - b).max() / (abs(K).sum(axis=1).max() * np.abs(xs).max())
    assert res <= 1e-10
