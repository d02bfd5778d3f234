"""Batched factorization: independent problems of uneven size factored and
solved together in one launch per tree level, each with the inertia the
reference gives for it alone and a residual <= 1e-10, and identical to the
same problem factored alone."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from amigo_b200 import linalg
from matrices import csr_arrays, kkt_matrix

pytestmark = pytest.mark.gpu


def test_batched_matches_single_and_reference(oracle_ref):
    r = np.random.RandomState(0)
    mats = [kkt_matrix(int(a), int(min(b, a - 5)), 300 + i)
            for i, (a, b) in enumerate(zip(r.randint(20, 400, 12),
                                           r.randint(10, 200, 12)))]
    mats = [M for M in mats if M.shape[0] > 0]
    pats = [csr_arrays(M)[:3] for M in mats]
    B = linalg.BatchedSparseLDL(pats, order=linalg.OrderingType.AMD,
                                device="cuda:0")
    vals = torch.from_numpy(np.concatenate([M.data for M in mats])).cuda()
    B.factor(vals)
    inertia = B.get_inertia()
    rhs = [M @ r.randn(M.shape[0]) for M in mats]
    x = torch.from_numpy(np.concatenate(rhs)).cuda()
    B.solve_device(x)
    xh = x.cpu().numpy()
    for i, M in enumerate(mats):
        n, rp, ci, v = csr_arrays(M)
        R = oracle_ref.RefSparseLDL(n, rp, ci, order="AMD")
        R.factor(v)
        assert inertia[i] == R.inertia()
        xi = xh[B.var_off[i]:B.var_off[i + 1]]
        res = np.abs(M @ xi - rhs[i]).max() / (abs(M).sum(axis=1).max() *
                                               np.abs(xi).max())
        assert res <= 1e-10
        # the same problem alone gives the same solution
        mat = linalg.CSRMat(n, n, rp, ci, v)
        single = linalg.SparseLDL(mat, order=linalg.OrderingType.AMD)
        single.factor()
        assert single.get_inertia() == inertia[i]
        xs = rhs[i].copy()
        single.solve(xs)
        np.testing.assert_allclose(xs, xi, rtol=1e-12, atol=1e-14)
