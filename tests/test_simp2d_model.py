"""CPU checks of the 2D SIMP model restatement (oracle/simp2d_oracle.py):
gradient and Hessian against central finite differences of the Lagrangian,
KKT pattern invariants, and the configured sizes."""
import numpy as np
import scipy.sparse as sp

from amigo_b200.problems.simp2d import Simp2D
from oracle import simp2d_oracle as O


def rand_point(m, seed):
    r = np.random.RandomState(seed)
    x = r.randn(m.n) * 0.3
    x[m.rt0:m.rt0 + m.nnodes] = 0.2 + 0.6 * r.rand(m.nnodes)
    x[m.re0:m.re0 + m.nelems] = 0.2 + 0.6 * r.rand(m.nelems)
    return x


def test_config_sizes():
    m = Simp2D(128, 64)
    assert 2 * m.nnodes == 16770 and m.nelems == 8192 and m.nnodes == 8385
    assert m.n == 16770 + 8385 + 8192 + 1 + 16770 + 8385 + 1
    assert m.nnz > 2.0e6
    K = sp.csr_matrix((np.ones(m.nnz), m.cols, m.rowp), shape=(m.n, m.n))
    assert (K - K.T).nnz == 0  # symmetric pattern
    assert np.all(m.diag_pos >= 0)


def test_gradient_and_hessian_match_finite_differences():
    m = Simp2D(6, 3, seed=1)
    x = rand_point(m, 2)
    g = O.gradient(m, x, alpha=0.7)
    h = 1e-6
    r = np.random.RandomState(3)
    for i in r.choice(m.n, 60, replace=False):
        e = np.zeros(m.n)
        e[i] = h
        fd = (O.lagrangian(m, x + e, 0.7) - O.lagrangian(m, x - e, 0.7)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), i
    # Hessian columns (without the fixed-row treatment)
    H, Fb = O.hessian_dense_blocks(m, x)
    vals = np.zeros(m.nnz)
    np.add.at(vals, m.epos.ravel(), H.reshape(-1))
    np.add.at(vals, m.fpos.ravel(), np.broadcast_to(Fb.ravel(), (m.nelems, 81)).ravel())
    np.add.at(vals, m.vpos.ravel(), 1.0 / m.nelems)
    np.add.at(vals, m.spos, -1.0)
    K = sp.csr_matrix((vals, m.cols, m.rowp), shape=(m.n, m.n)).toarray()
    for i in r.choice(m.n, 60, replace=False):
        e = np.zeros(m.n)
        e[i] = h
        fd = (O.gradient(m, x + e, 0.7) - O.gradient(m, x - e, 0.7)) / (2 * h)
        assert np.abs(fd - K[:, i]).max() <= 1e-6 * max(1.0, np.abs(K[:, i]).max()), i


def test_fixed_rows_unit_diagonal():
    m = Simp2D(8, 4)
    x = rand_point(m, 5)
    K = sp.csr_matrix((O.hessian_values(m, x), m.cols, m.rowp), shape=(m.n, m.n))
    Kd = K.toarray()
    for i in m.fixed:
        row = Kd[i].copy()
        assert row[i] == 1.0
        row[i] = 0.0
        assert not row.any() and not np.delete(Kd[:, i], i).any()
