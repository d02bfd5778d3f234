"""Large-front panels on a thread-block cluster (8 CTAs per front) against
the one-CTA panel.  With the one-CTA panel's widths (panel mode 2) the
cluster panel reproduces the one-CTA panel (mode 1) bit for bit -- inertia,
per-node pivot and delay counts and the solution of a solve -- since every
row's arithmetic, the reductions and the pivot decisions are the same.
With full-width panels (mode 0, the default) the factor is a different
rounding of the same algorithm: identical inertia, per-node pivot counts
equal on >= 90% of the nodes, relative residual <= 1e-10.  The
global-scratch form (W and L in HBM/L2, clusters of 16 CTAs; panel mode 3)
reproduces mode 0 bit for bit, and on 3D fronts past shared memory (mode 0
switches to it by itself) it agrees with the one-CTA panel to rounding."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from matrices import csr_arrays, kkt_matrix

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ldl_golden.npz")


def rel_residual(K, x, b):
    r = K @ x - b
    return np.abs(r).max() / (abs(K).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())


def factor_solve(K, mode, min_rows, precision=64, order=None, ustab=0.01):
    from amigo_b200 import linalg
    n, rp, ci, v = csr_arrays(K)
    mat = linalg.CSRMat(n, n, rp, ci, v)
    ldl = linalg.SparseLDL(mat, ustab=ustab,
                           order=linalg.OrderingType.AMD if order is None else order)
    ldl.set_panel_mode(mode, min_rows)
    if precision != 64:
        ldl.set_precision(precision)
    assert ldl.factor() == 0
    b = K @ np.random.RandomState(5).randn(n)
    x = b.copy()
    ldl.solve(x)
    npiv, ndel = ldl.node_pivots()
    return ldl.get_inertia(), npiv, ndel, x, b


def simp_kkt(nx, ny, seed=3):
    from amigo_b200.problems.simp2d import Simp2D
    from oracle import simp2d_oracle as O
    m = Simp2D(nx, ny, seed=seed)
    vals = O.hessian_values(m, m.initial_point())
    prim = ~m.mult
    d = np.zeros(m.n)
    d[prim] = 1e-2 + np.random.RandomState(1).rand(prim.sum())
    vals[m.diag_pos] += d
    vals[m.fixed_diag_pos] = 1.0
    return sp.csr_matrix((vals, m.cols, m.rowp), shape=(m.n, m.n))


def check(K, min_rows, precision=64, **kw):
    i1, p1, d1, x1, b = factor_solve(K, 1, min_rows, precision, **kw)
    i2, p2, d2, x2, _ = factor_solve(K, 2, min_rows, precision, **kw)
    assert i2 == i1
    assert np.array_equal(p2, p1) and np.array_equal(d2, d1)
    assert np.array_equal(x2, x1), np.abs(x2 - x1).max()
    i0, p0, d0, x0, _ = factor_solve(K, 0, min_rows, precision, **kw)
    assert i0 == i1
    assert np.mean(p0 == p1) >= 0.9
    bar = 1e-10 if precision == 64 else 1e-4
    assert rel_residual(K, x0, b) <= bar
    assert rel_residual(K, x1, b) <= bar


def test_golden_fixtures_every_large_level_on_clusters():
    z = np.load(GOLD)
    for name in sorted({k.split("/")[0] for k in z.files}):
        rp, ci, v = z[name + "/rowp"], z[name + "/cols"], z[name + "/vals"]
        n = len(rp) - 1
        K = sp.csr_matrix((v, ci, rp), shape=(n, n))
        check(K, 1, order=int(z[name + "/order"]), ustab=float(z[name + "/ustab"]))


@pytest.mark.parametrize("seed", [11, 12])
def test_kkt_with_delays(seed):
    K = kkt_matrix(2500, 1200, seed)
    check(K, 1)


def test_simp2d_64x32():
    check(simp_kkt(64, 32), 1)


def test_simp2d_64x32_fp32():
    check(simp_kkt(64, 32), 1, precision=32)


def test_simp2d_128x64_default_threshold():
    check(simp_kkt(128, 64), 0)


def check_global_form(K, min_rows, precision=64):
    i0, p0, d0, x0, b = factor_solve(K, 0, min_rows, precision)
    i3, p3, d3, x3, _ = factor_solve(K, 3, min_rows, precision)
    assert i3 == i0
    assert np.array_equal(p3, p0) and np.array_equal(d3, d0)
    assert np.array_equal(x3, x0), np.abs(x3 - x0).max()


def test_global_scratch_form_simp2d_128x64():
    check_global_form(simp_kkt(128, 64), 1)


def test_global_scratch_form_with_delays():
    check_global_form(kkt_matrix(2500, 1200, 11), 1)


def test_global_scratch_form_fp32():
    check_global_form(simp_kkt(64, 32), 1, precision=32)


def simp3d_kkt(nx, ny, nz, seed=3):
    from amigo_b200.problems.simp3d import Simp3D
    m = Simp3D(nx, ny, nz, seed=seed)
    rp, ci = m.rowp, m.cols
    rng = np.random.RandomState(seed)
    n = m.n
    # a quasi-definite KKT on the pattern: SPD primal block, negative
    # diagonal on the multiplier rows
    A = sp.csr_matrix((rng.randn(len(ci)) * 0.1, ci, rp), shape=(n, n))
    A = (A + A.T) * 0.5
    d = np.where(m.mult, -1.0, 1.0) * (1.0 + abs(A).sum(axis=1).A1)
    K = sp.csr_matrix(A + sp.diags(d))
    K.sort_indices()
    return K


def test_simp3d_large_fronts_global_form():
    K = simp3d_kkt(20, 10, 10)
    i1, p1, d1, x1, b = factor_solve(K, 1, 1)
    i0, p0, d0, x0, _ = factor_solve(K, 0, 0)
    assert i0 == i1
    assert rel_residual(K, x0, b) <= 1e-10
    assert rel_residual(K, x1, b) <= 1e-10
