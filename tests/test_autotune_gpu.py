"""The autotuner (ab_ldl_autotune): it times the large-front panel forms and
the solve schedules on the caller's KKT and keeps the fastest.  Whatever it
picks, the factorization is the same algorithm to rounding -- identical
inertia, per-node pivot counts equal on >= 90% of the nodes, relative
residual <= 1e-10 -- the solve thresholds change the solution only to
rounding (relative residual <= 1e-10) and the narrow-front schedules not at
all.  Stored settings are reused for a second handle of the same pattern."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from matrices import csr_arrays, kkt_matrix

pytestmark = pytest.mark.gpu

DEFAULT_PANEL = dict(panel_mode=0, cl_min_rows=768, panel_cache_bytes=0)


def rel_residual(K, x, b):
    r = K @ x - b
    return np.abs(r).max() / (abs(K).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())


def simp_kkt(nx, ny):
    from amigo_b200.problems.simp2d import Simp2D
    from oracle import simp2d_oracle as O
    m = Simp2D(nx, ny, seed=3)
    vals = O.hessian_values(m, m.initial_point())
    prim = ~m.mult
    d = np.zeros(m.n)
    d[prim] = 1e-2 + np.random.RandomState(1).rand(prim.sum())
    vals[m.diag_pos] += d
    vals[m.fixed_diag_pos] = 1.0
    return sp.csr_matrix((vals, m.cols, m.rowp), shape=(m.n, m.n))


def make(K):
    from amigo_b200 import linalg
    n, rp, ci, v = csr_arrays(K)
    mat = linalg.CSRMat(n, n, rp, ci, v)
    return linalg.SparseLDL(mat, order=linalg.OrderingType.AMD)


def solve(ldl, b):
    x = b.copy()
    ldl.solve(x)
    return x


def apply(ldl, t):
    from amigo_b200 import _lib, linalg
    s = linalg.LdlTuning()
    for k, _ in s._fields_:
        if k in t:
            setattr(s, k, t[k])
    _lib.call("ab_ldl_apply_tuning", ldl._h, ctypes.byref(s))


@pytest.mark.parametrize("shape", [(64, 32), (128, 64)])
def test_tuned_factor_is_the_same_factorization(shape):
    K = simp_kkt(*shape)
    b = K @ np.random.RandomState(5).randn(K.shape[0])
    ref = make(K)
    assert ref.factor() == 0
    x0 = solve(ref, b)
    p0, _ = ref.node_pivots()

    ldl = make(K)
    t = ldl.autotune(reps=2, cache=False)
    assert not t["cached"] and t["configurations"] >= 2
    assert 0.0 < t["factor_ms"] <= t["factor_ms_initial"]
    assert 0.0 < t["solve_ms"] <= t["solve_ms_initial"]
    # left factored with the chosen settings
    assert ldl.get_inertia() == ref.get_inertia()
    x = solve(ldl, b)
    assert rel_residual(K, x, b) <= 1e-10
    p, _ = ldl.node_pivots()
    assert (p == p0).mean() >= 0.9
    ldl.solve_status()

    # the solve settings alone on the default factorization: a solution to
    # rounding, and the narrow-front schedule alone the same bits
    same = make(K)
    apply(same, dict(t, **DEFAULT_PANEL))
    assert same.factor() == 0
    assert same.get_inertia() == ref.get_inertia()
    assert rel_residual(K, solve(same, b), b) <= 1e-10
    q = make(K)
    q.set_solve_queue(t["solve_queue"])
    assert q.factor() == 0
    assert np.array_equal(solve(q, b), x0)


def test_settings_reused_for_the_same_pattern():
    from amigo_b200 import linalg
    K = simp_kkt(32, 16)
    linalg._TUNED.clear()
    a = make(K).autotune(reps=1)
    second = make(K)
    c = second.autotune(reps=1)
    assert not a["cached"] and c["cached"]
    for k in ("panel_mode", "cl_min_rows", "cluster_entries", "wide_entries", "solve_queue"):
        assert a[k] == c[k]
    b = K @ np.ones(K.shape[0])
    assert rel_residual(K, solve(second, b), b) <= 1e-10


def test_batched_handle():
    """Small fronts only: the factorization is the untuned one (same
    inertia), the solutions agree to rounding."""
    from amigo_b200 import linalg
    r = np.random.RandomState(0)
    mats = [kkt_matrix(int(a), int(min(c, a - 5)), 700 + i)
            for i, (a, c) in enumerate(zip(r.randint(20, 400, 10), r.randint(10, 200, 10)))]
    pats = [csr_arrays(M)[:3] for M in mats]
    vals = torch.from_numpy(np.concatenate([M.data for M in mats])).cuda()
    rhs = np.concatenate([M @ r.randn(M.shape[0]) for M in mats])

    def run(tune):
        B = linalg.BatchedSparseLDL(pats, order=linalg.OrderingType.AMD, device="cuda:0")
        if tune:
            t = B.autotune(vals, reps=1, cache=False)
            assert t["configurations"] >= 2
        else:
            B.factor(vals)
        x = torch.from_numpy(rhs.copy()).cuda()
        B.solve_device(x)
        return B.get_inertia(), x.cpu().numpy()

    i0, x0 = run(False)
    i1, x1 = run(True)
    assert i0 == i1
    off = np.concatenate([[0], np.cumsum([M.shape[0] for M in mats])])
    for k, M in enumerate(mats):
        b = rhs[off[k]:off[k + 1]]
        for x in (x0, x1):
            assert rel_residual(M, x[off[k]:off[k + 1]], b) <= 1e-10


def test_arguments():
    from amigo_b200 import _lib, linalg
    lib = _lib.lib()
    assert lib.ab_ldl_autotune(None, None, 1, None, None) == -1
    ldl = make(simp_kkt(8, 4))
    assert lib.ab_ldl_autotune(ldl._h, ldl.mat.vals.data_ptr(), 0, None, None) == -1
    bad = linalg.LdlTuning(panel_mode=7, cl_min_rows=768, cluster_entries=1,
                           wide_entries=1)
    assert lib.ab_ldl_apply_tuning(ldl._h, ctypes.byref(bad)) == -1
