"""Mixed-precision factorization (FP32 fronts, FP64 pivot tests and solve
accumulation) with FP64 iterative refinement against the FP64 KKT.

Bar: on the fixtures the FP32-front factorization reports the same inertia
as the FP64 one, one FP32-factor solve has a relative residual of FP32
order (<= 1e-4) and refinement with the FP64 matrix brings it to the FP64
bar <= 1e-10 within 10 steps.  The 2D SIMP KKT (Emin = 1e-9) has
eigenvalues below FP32 resolution: its FP32 inertia may move by a few
pivots, and then the mixed-precision backend must notice and refactor in
FP64 (the test checks that it does and that the result meets the FP64
bar)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from matrices import csr_arrays, kkt_matrix

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ldl_golden.npz")


def rel_residual(K, x, b):
    r = K @ x - b
    kn = abs(K).sum(axis=1).max()
    return np.abs(r).max() / (kn * np.abs(x).max() + np.abs(b).max())


def refine(mat, ldl, b, steps=10, tol=1e-12):
    """x = K^-1 b by the FP32 factor plus classic refinement with the FP64
    matrix on the device; returns x and the steps taken."""
    x = b.clone()
    ldl.solve_device(x)
    r = torch.empty_like(b)
    for k in range(steps):
        mat.mult(x, r)
        r.sub_(b).neg_()
        if r.abs().max().item() <= tol * b.abs().max().item():
            return x, k
        ldl.solve_device(r)
        x.add_(r)
    return x, steps


def factor_both(M, order):
    from amigo_b200 import linalg
    n, rp, ci, v = csr_arrays(M)
    mat = linalg.CSRMat(n, n, rp, ci, v)
    l64 = linalg.SparseLDL(mat, order=order)
    l64.factor()
    l32 = linalg.SparseLDL(mat, order=order, precision="fp32")
    l32.factor()
    return mat, l64, l32


@pytest.mark.parametrize("case", ["kkt700_AMD", "kkt200_AMD", "poisson20_AMD",
                                  "kkt700_NESTED_DISSECTION"])
def test_golden_inertia_and_refinement(case):
    z = np.load(GOLD)
    rp, ci, v = z[case + "/rowp"], z[case + "/cols"], z[case + "/vals"]
    n = len(rp) - 1
    M = sp.csr_matrix((v, ci, rp), shape=(n, n))
    mat, l64, l32 = factor_both(M, int(z[case + "/order"]))
    assert l32.get_inertia() == l64.get_inertia() == tuple(z[case + "/inertia"])
    bh = M @ np.random.RandomState(0).randn(n)
    b = torch.from_numpy(bh).cuda()
    x1 = b.clone()
    l32.solve_device(x1)
    assert rel_residual(M, x1.cpu().numpy(), bh) <= 1e-4
    x, steps = refine(mat, l32, b)
    assert rel_residual(M, x.cpu().numpy(), bh) <= 1e-10
    assert steps <= 10


def test_simp2d_kkt_mixed():
    """The 2D SIMP KKT with a quasi-definite diagonal (inertia known:
    (primal rows, multiplier rows)).  Either the FP32-front factor has that
    inertia and refinement against the FP64 matrix reaches 1e-10, or the
    mixed-precision backend detects the mismatch and refactors in FP64, whose
    inertia is exact and whose refined solve meets the same bar."""
    from amigo_b200.ipm_driver import DeviceBackend, SimpProblem
    from amigo_b200.problems.simp2d import Simp2D
    m = Simp2D(64, 32, seed=3)
    B = DeviceBackend(SimpProblem(m, "cuda:0"), m, "cuda:0", precision="fp32")
    st = B.initial_state()
    prim = torch.from_numpy(~m.mult).cuda()
    g = torch.Generator(device="cuda:0").manual_seed(1)
    diag = torch.where(prim, 1e-2 + torch.rand(m.n, dtype=torch.float64, device="cuda:0",
                                               generator=g), 0.0)
    inertia = B.factor(st, diag, 0.0, 0.0)
    assert inertia == (B.np, B.nc)
    assert B.fp64_now == (B.inertia_fallbacks > 0)
    K = B.solver.hess
    _, _, _, rp, ci = K.get_nonzero_structure()
    vals = K.vals.cpu().numpy()
    M = sp.csr_matrix((vals, np.asarray(ci), np.asarray(rp)), shape=(m.n, m.n))
    bh = M @ np.random.RandomState(2).randn(m.n)
    b = torch.from_numpy(bh).cuda()
    x, steps = refine(K, B.solver.ldl, b, steps=20)
    assert rel_residual(M, x.cpu().numpy(), bh) <= 1e-10
