"""CPU checks of the 3D SIMP model (problems/simp3d.py) and of the
dimension-generic restatement oracle/simp2d_oracle.py on it: element
matrices, gradient and Hessian against central finite differences of the
Lagrangian, pattern invariants, and the configured sizes."""
import numpy as np
import scipy.sparse as sp

from amigo_b200.problems.simp3d import Simp3D, element_matrices
from oracle import simp2d_oracle as O


def rand_point(m, seed):
    r = np.random.RandomState(seed)
    x = r.randn(m.n) * 0.3
    x[m.rt0:m.rt0 + m.nnodes] = 0.2 + 0.6 * r.rand(m.nnodes)
    x[m.re0:m.re0 + m.nelems] = 0.2 + 0.6 * r.rand(m.nelems)
    return x


def test_element_matrices():
    K0, M, KL = element_matrices()
    assert np.abs(K0 - K0.T).max() < 1e-15
    ev = np.linalg.eigvalsh(K0)
    assert np.all(np.abs(ev[:6]) < 1e-12) and ev[6] > 1e-3   # 6 rigid modes
    assert abs(M.sum() - 1.0) < 1e-14                          # unit volume
    assert np.abs(KL.sum(axis=1)).max() < 1e-14                # constants in null space


def test_config_sizes():
    nx, ny, nz = 48, 24, 24
    nn = (nx + 1) * (ny + 1) * (nz + 1)
    ne = nx * ny * nz
    assert 3 * nn == 91875 and ne == 27648 and nn == 30625
    assert 3 * nn + nn + ne + 1 + 3 * nn + nn + 1 == 272650
    m = Simp3D(6, 3, 3)
    nn, ne = 7 * 4 * 4, 6 * 3 * 3
    assert m.n == 3 * nn + nn + ne + 1 + 3 * nn + nn + 1
    K = sp.csr_matrix((np.ones(m.nnz), m.cols, m.rowp), shape=(m.n, m.n))
    assert (K - K.T).nnz == 0
    assert np.all(m.diag_pos >= 0)
    assert len(m.fixed) == 2 * 3 * 4 * 4
    assert abs(m.f.sum() + 1.0) < 1e-15                       # unit total load


def test_gradient_and_hessian_match_finite_differences():
    m = Simp3D(3, 2, 2, seed=1)
    x = rand_point(m, 2)
    g = O.gradient(m, x, alpha=0.7)
    h = 1e-6
    r = np.random.RandomState(3)
    for i in r.choice(m.n, 60, replace=False):
        e = np.zeros(m.n)
        e[i] = h
        fd = (O.lagrangian(m, x + e, 0.7) - O.lagrangian(m, x - e, 0.7)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), i
    H, Fb = O.hessian_dense_blocks(m, x)
    vals = np.zeros(m.nnz)
    np.add.at(vals, m.epos.ravel(), H.reshape(-1))
    np.add.at(vals, m.fpos.ravel(), np.broadcast_to(Fb.ravel(), (m.nelems, Fb.size)).ravel())
    np.add.at(vals, m.vpos.ravel(), 1.0 / m.nelems)
    np.add.at(vals, m.spos, -1.0)
    K = sp.csr_matrix((vals, m.cols, m.rowp), shape=(m.n, m.n)).toarray()
    for i in r.choice(m.n, 60, replace=False):
        e = np.zeros(m.n)
        e[i] = h
        fd = (O.gradient(m, x + e, 0.7) - O.gradient(m, x - e, 0.7)) / (2 * h)
        assert np.abs(fd - K[:, i]).max() <= 1e-6 * max(1.0, np.abs(K[:, i]).max()), i
