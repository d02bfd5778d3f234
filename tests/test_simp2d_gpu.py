"""GPU element kernels of the 2D SIMP model (gradient, Hessian scatter into
the CSR KKT values, fixed rows) against the numpy restatement
oracle/simp2d_oracle.py (itself pinned by finite differences).  FP64 with
different summation order: rtol 1e-13 relative to the largest entry."""
import numpy as np
import pytest
import torch

from amigo_b200.problems.simp2d import Simp2D
from oracle import simp2d_oracle as O

pytestmark = pytest.mark.gpu


def rand_point(m, seed):
    r = np.random.RandomState(seed)
    x = r.randn(m.n) * 0.3
    x[m.rt0:m.rt0 + m.nnodes] = 0.2 + 0.6 * r.rand(m.nnodes)
    x[m.re0:m.re0 + m.nelems] = 0.2 + 0.6 * r.rand(m.nelems)
    return x


@pytest.mark.parametrize("mesh", [(6, 3), (40, 20), (128, 64)])
def test_gradient_and_hessian(mesh):
    m = Simp2D(*mesh, seed=4)
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
    # deterministic: a second evaluation is bit-identical
    vals2 = torch.zeros_like(vals)
    dm.hessian(xd, 0.9, vals2)
    assert torch.equal(vals, vals2)


def test_kkt_factor_matches_reference(oracle_ref):
    import scipy.sparse as sp
    from amigo_b200 import linalg
    m = Simp2D(32, 16, seed=2)
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


def _bench_point_kkt(m, dev):
    """KKT values of the 2D SIMP model at its seeded initial point with the
    barrier diagonal of the first IPM iteration, assembled by the product's
    kernels (the benchmark's workload)."""
    from amigo_b200.ipm import InteriorPointOptimizer
    dm = m.device_model(dev)
    opt = InteriorPointOptimizer(m.mult, m.lower, m.upper, device=dev)
    opt.relax_bounds()
    x = torch.from_numpy(m.initial_point()).to(dev)
    v = opt.create_opt_vector(x)
    opt.initialize_multipliers_and_slacks(0.1, None, v)
    vals = torch.zeros(m.nnz, dtype=torch.float64, device=dev)
    dm.hessian(v.x, 1.0, vals)
    diag = torch.zeros(m.n, dtype=torch.float64, device=dev)
    opt.compute_diagonal(v, diag)
    diag += 1e-8 * torch.from_numpy((~m.mult).astype(np.float64)).to(dev)
    vals[torch.from_numpy(m.diag_pos.astype(np.int64)).to(dev)] += diag
    return vals.cpu().numpy()


def _compare_with_reference(oracle_ref, m, vals, min_equal=0.9):
    import scipy.sparse as sp
    from amigo_b200 import linalg
    R = oracle_ref.RefSparseLDL(m.n, m.rowp, m.cols, order="AMD")
    R.factor(vals)
    mat = linalg.CSRMat(m.n, m.n, m.rowp, m.cols, vals)
    ldl = linalg.SparseLDL(mat, order=linalg.OrderingType.AMD)
    ldl.factor()
    assert ldl.get_inertia() == R.inertia()
    npiv, ndel = ldl.node_pivots()
    rpiv, rdel = R.node_pivots()
    assert np.mean(npiv == rpiv) >= min_equal, np.mean(npiv == rpiv)
    K = sp.csr_matrix((vals, m.cols, m.rowp), shape=(m.n, m.n))
    b = K @ np.random.RandomState(3).randn(m.n)
    xg = b.copy()
    ldl.solve(xg)
    r = np.abs(K @ xg - b).max() / (abs(K).sum(axis=1).max() * np.abs(xg).max())
    assert r <= 1e-10, r
    return ldl, R


def test_kkt_128x64_bench_point_matches_reference(oracle_ref):
    """The benchmarked 128 x 64 KKT (n = 58,504): the same values factored by
    the reference's SparseLDL on the host and by the GPU: identical inertia,
    >= 90% identical per-node pivot counts, relative residual <= 1e-10."""
    m = Simp2D(128, 64)
    vals = _bench_point_kkt(m, "cuda:0")
    _compare_with_reference(oracle_ref, m, vals)
