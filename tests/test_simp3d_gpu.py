"""GPU element kernels of the 3D SIMP model (trilinear hexahedra: gradient,
Hessian scatter into the CSR KKT values, fixed rows) against the numpy
restatement oracle/simp2d_oracle.py (dimension-generic, pinned by finite
differences in tests/test_simp3d_model.py), and a KKT factorization of a
small 3D cantilever against the reference's own SparseLDL.  FP64 with
different summation order: rtol 1e-13 relative to the largest entry."""
import numpy as np
import pytest
import torch

from amigo_b200.problems.simp3d import Simp3D
from oracle import simp2d_oracle as O

pytestmark = pytest.mark.gpu


def rand_point(m, seed):
    r = np.random.RandomState(seed)
    x = r.randn(m.n) * 0.3
    x[m.rt0:m.rt0 + m.nnodes] = 0.2 + 0.6 * r.rand(m.nnodes)
    x[m.re0:m.re0 + m.nelems] = 0.2 + 0.6 * r.rand(m.nelems)
    return x


@pytest.mark.parametrize("mesh", [(4, 2, 2), (12, 6, 6)])
def test_gradient_and_hessian(mesh):
    m = Simp3D(*mesh, seed=4)
    dm = m.device_model("cuda:0")
    x = rand_point(m, 11)
    xd = torch.from_numpy(x).cuda()
    g = torch.zeros(m.n, dtype=torch.float64, device="cuda:0")
    dm.gradient(xd, 0.9, g)
    want = O.gradient_fixed(m, x, 0.9)
    got = g.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * max(1.0, np.abs(want).max())
    vals = torch.full((m.nnz,), 7.0, dtype=torch.float64, device="cuda:0")
    dm.hessian(xd, 0.9, vals)
    want = O.hessian_values(m, x)
    got = vals.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * max(1.0, np.abs(want).max())
    vals2 = torch.zeros_like(vals)
    dm.hessian(xd, 0.9, vals2)
    assert torch.equal(vals, vals2)


def test_kkt_factor_matches_reference(oracle_ref):
    import scipy.sparse as sp
    from amigo_b200 import linalg
    m = Simp3D(8, 4, 4, seed=2)
    x = m.initial_point()
    vals = O.hessian_values(m, x)
    prim = ~m.mult
    d = np.zeros(m.n)
    d[prim] = 1.0 + np.random.RandomState(0).rand(prim.sum())
    vals[m.diag_pos] += d
    vals[m.fixed_diag_pos] = 1.0
    K = sp.csr_matrix((vals, m.cols, m.rowp), shape=(m.n, m.n))
    R = oracle_ref.RefSparseLDL(m.n, m.rowp, m.cols, order="AMD")
    R.factor(vals)
    mat = linalg.CSRMat(m.n, m.n, m.rowp, m.cols, vals)
    ldl = linalg.SparseLDL(mat, order=linalg.OrderingType.AMD)
    ldl.factor()
    assert ldl.get_inertia() == R.inertia()
    b = K @ np.random.RandomState(1).randn(m.n)
    xg = b.copy()
    ldl.solve(xg)
    r = np.abs(K @ xg - b).max() / (abs(K).sum(axis=1).max() * np.abs(xg).max())
    assert r <= 1e-10
