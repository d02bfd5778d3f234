"""The multi-CTA solves against the one-CTA-per-front solve: every golden
fixture and a 2D SIMP KKT are solved with all fronts on the cooperative
wide path (wide threshold 1), with every front on one CTA (both thresholds
2^62), with every front on the cluster path (cluster threshold 1, wide
2^62), and with the default split.  Each meets the FP64 residual bar 1e-10; the solutions
differ only by summation order (1e-9 relative on the fixtures, 1e-6 on the
ill-conditioned SIMP KKT).  Also several right-hand sides at once."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from matrices import csr_arrays

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ldl_golden.npz")


def rel_residual(K, x, b):
    r = K @ x - b
    kn = abs(K).sum(axis=1).max()
    return np.abs(r).max() / (kn * np.abs(x).max() + np.abs(b).max())


def solve_three_ways(M, order, ustab=0.01, nrhs=1):
    from amigo_b200 import linalg
    n, rp, ci, v = csr_arrays(M)
    mat = linalg.CSRMat(n, n, rp, ci, v)
    ldl = linalg.SparseLDL(mat, ustab=ustab, order=order)
    assert ldl.factor() == 0
    B = (M @ np.random.RandomState(7).randn(n, nrhs)).T.copy()   # nrhs x n
    out = []
    for clu, wide in ((1 << 62, 1), (1 << 62, 1 << 62), (1, 1 << 62), (1 << 14, 1 << 22)):
        ldl.set_cluster_threshold(clu)
        ldl.set_wide_threshold(wide)
        xd = torch.from_numpy(B.copy()).cuda()
        ldl.solve_device(xd if nrhs > 1 else xd[0])
        out.append(xd.cpu().numpy())
    return B, out


def test_golden_cases_wide_equals_narrow():
    z = np.load(GOLD)
    names = sorted({k.split("/")[0] for k in z.files})
    for name in names:
        rp, ci, v = z[name + "/rowp"], z[name + "/cols"], z[name + "/vals"]
        n = len(rp) - 1
        M = sp.csr_matrix((v, ci, rp), shape=(n, n))
        B, (xw, xn, xc, xd) = solve_three_ways(M, int(z[name + "/order"]),
                                               float(z[name + "/ustab"]))
        scale = np.abs(xn).max()
        assert np.abs(xw - xn).max() <= 1e-9 * scale, name
        assert np.abs(xc - xn).max() <= 1e-9 * scale, name
        assert np.abs(xd - xn).max() <= 1e-9 * scale, name
        for x in (xw, xn, xc, xd):
            assert rel_residual(M, x[0], B[0]) <= 1e-10, name


def test_simp2d_kkt_wide_fronts_multi_rhs():
    from amigo_b200 import linalg
    from amigo_b200.problems.simp2d import Simp2D
    from oracle import simp2d_oracle as O
    m = Simp2D(64, 32, seed=3)
    vals = O.hessian_values(m, m.initial_point())
    prim = ~m.mult
    d = np.zeros(m.n)
    d[prim] = 1e-2 + np.random.RandomState(1).rand(prim.sum())
    vals[m.diag_pos] += d
    vals[m.fixed_diag_pos] = 1.0
    M = sp.csr_matrix((vals, m.cols, m.rowp), shape=(m.n, m.n))
    B, (xw, xn, xc, xd) = solve_three_ways(M, linalg.OrderingType.AMD, nrhs=3)
    for x in (xw, xn, xc, xd):
        for k in range(3):
            assert rel_residual(M, x[k], B[k]) <= 1e-10
    # Emin = 1e-9 makes this KKT ill-conditioned: solutions of equal
    # residual differ at the 1e-8 level
    scale = np.abs(xn).max()
    assert np.abs(xw - xn).max() <= 1e-6 * scale
    assert np.abs(xc - xn).max() <= 1e-6 * scale
    assert np.abs(xd - xn).max() <= 1e-6 * scale
