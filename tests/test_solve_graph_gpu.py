"""Solves captured as CUDA graphs (linalg.SolveGraph): a replay gives the
eager solve's bits, every replay is a fresh work-queue sweep (the sweep
epoch lives in device memory), and a new factorization is captured again."""
import numpy as np
import pytest
import torch

from matrices import csr_arrays, kkt_matrix
from test_autotune_gpu import simp_kkt

pytestmark = pytest.mark.gpu


def eager(ldl, b):
    x = torch.from_numpy(b.copy()).cuda()
    ldl.solve_device(x)
    return x.cpu().numpy()


@pytest.mark.parametrize("wide", [None, 1 << 16])
def test_simp2d_replays_match_eager(wide):
    from amigo_b200 import linalg
    K = simp_kkt(64, 32)
    n, rp, ci, v = csr_arrays(K)
    mat = linalg.CSRMat(n, n, rp, ci, v)
    ldl = linalg.SparseLDL(mat, order=linalg.OrderingType.AMD)
    if wide is not None:
        ldl.set_wide_threshold(wide)   # cooperative grid kernels in the graph
    ldl.factor()
    b = K @ np.random.RandomState(2).randn(n)
    x0 = eager(ldl, b)
    xd = torch.empty(n, dtype=torch.float64, device="cuda")
    g = linalg.SolveGraph(ldl, xd)
    for _ in range(3):
        xd.copy_(torch.from_numpy(b))
        g()
        assert np.array_equal(xd.cpu().numpy(), x0)
    assert g.captures == 1 and g.replays == 3
    # a new factorization: captured again
    mat.vals.mul_(2.0)
    ldl.factor()
    x1 = eager(ldl, b)
    xd.copy_(torch.from_numpy(b))
    g()
    assert g.captures == 2
    assert np.array_equal(xd.cpu().numpy(), x1)
    ldl.solve_status()


def test_batched_queue_sweeps_replay():
    """Many small fronts: the sweeps are work-queue launches whose waits
    compare done flags with the sweep's epoch."""
    from amigo_b200 import linalg
    r = np.random.RandomState(4)
    mats = [kkt_matrix(int(a), int(min(c, a - 5)), 900 + i)
            for i, (a, c) in enumerate(zip(r.randint(20, 300, 16), r.randint(10, 150, 16)))]
    pats = [csr_arrays(M)[:3] for M in mats]
    vals = torch.from_numpy(np.concatenate([M.data for M in mats])).cuda()
    B = linalg.BatchedSparseLDL(pats, order=linalg.OrderingType.AMD, device="cuda:0")
    B.factor(vals)
    xd = torch.empty(B.n, dtype=torch.float64, device="cuda")
    g = linalg.SolveGraph(B, xd)
    for k in range(4):
        b = np.random.RandomState(10 + k).randn(B.n)
        ref = torch.from_numpy(b.copy()).cuda()
        B.solve_device(ref)
        xd.copy_(torch.from_numpy(b))
        g()
        assert np.array_equal(xd.cpu().numpy(), ref.cpu().numpy())
    assert g.captures == 1
    B.solve_status()
