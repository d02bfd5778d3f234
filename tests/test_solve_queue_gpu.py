"""Narrow-front solve schedules against one another: one launch per level
or one work-queue launch per sweep (over the levels whose fronts are all
narrow), each with 256-thread CTAs for every front or 128-thread CTAs for
the fronts of at most 128 rows.  The per-front arithmetic and the order of the children's update
vectors are the same in all four, so the solutions agree bit for bit -- on
seeded KKT systems (one and several right-hand sides) and on a batch of
cart-pole KKT systems (every level narrow, every front small)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from matrices import csr_arrays, kkt_matrix

pytestmark = pytest.mark.gpu


def solve_both(ldl, b, n):
    """Solutions with schedule modes 0 (per level, CTA fronts) and 3 (queue,
    warp fronts); modes 1 and 2 must equal them too."""
    out = []
    for mode in (0, 1, 2, 3):
        ldl.set_solve_queue(mode)
        x = b.clone()
        ldl.solve_device(x)
        torch.cuda.synchronize()
        out.append(x.cpu().numpy())
    ldl.solve_status()
    for y in out[1:3]:
        assert np.array_equal(y, out[0])
    return out[0], out[3]


def test_single_kkt_queue_equals_levels():
    from amigo_b200 import linalg
    K = kkt_matrix(3000, 1400, 21)
    n, rp, ci, v = csr_arrays(K)
    mat = linalg.CSRMat(n, n, rp, ci, v)
    ldl = linalg.SparseLDL(mat)
    assert ldl.factor() == 0
    b = torch.from_numpy(np.random.RandomState(2).randn(n)).cuda()
    x0, x1 = solve_both(ldl, b, n)
    assert np.array_equal(x0, x1)
    r = K @ x1 - b.cpu().numpy()
    assert np.abs(r).max() <= 1e-10 * (abs(K).sum(axis=1).max() * np.abs(x1).max())


def test_multiple_rhs_queue_equals_levels():
    from amigo_b200 import linalg
    K = kkt_matrix(1500, 700, 4)
    n, rp, ci, v = csr_arrays(K)
    mat = linalg.CSRMat(n, n, rp, ci, v)
    ldl = linalg.SparseLDL(mat)
    assert ldl.factor() == 0
    b = torch.from_numpy(np.random.RandomState(3).randn(3, n)).cuda()
    x0, x1 = solve_both(ldl, b, n)
    assert np.array_equal(x0, x1)


def test_batched_cartpole_queue_equals_levels():
    from amigo_b200 import linalg
    from amigo_b200.problems.cartpole import batch_config
    B = batch_config(k=24, seed=7, nmin=50, nmax=200)
    pats = [(mm.n, mm.rowp, mm.cols) for mm in B.inst]
    ldl = linalg.BatchedSparseLDL(pats, device="cuda:0")
    vals = []
    for mm in B.inst:
        # a quasi-definite matrix on the instance's KKT pattern: symmetric
        # off-diagonal values, a dominant diagonal, negative on multipliers
        n = mm.n
        rr = np.repeat(np.arange(n), np.diff(mm.rowp))
        v = 0.1 * np.cos(0.37 * (rr + mm.cols))
        off = rr != mm.cols
        rowsum = np.bincount(rr[off], weights=np.abs(v[off]), minlength=n)
        dg = ~off
        v[dg] = np.where(mm.mult[rr[dg]], -1.0, 1.0) * (1.0 + rowsum[rr[dg]])
        vals.append(v)
    ldl.factor(torch.from_numpy(np.concatenate(vals)).cuda())
    b = torch.from_numpy(np.random.RandomState(1).randn(ldl.n)).cuda()
    x0, x1 = solve_both(ldl, b, ldl.n)
    assert np.array_equal(x0, x1)
    assert np.isfinite(x1).all()
