"""Batched interior-point solves: many cart-pole instances of uneven size
(N ~ U{50..150} here; the batched-trajectories config draws N ~ U{50..400},
pole mass ~ U(0.1, 0.5), final position ~ U(-1, 1)) solved together, each
phase one launch over all instances.  Bar: every instance converges with the
iteration count it takes when solved alone, the same objective to 1e-9
relative and the same optimum to 1e-7 (per-instance sums are taken in a
different order than the single-problem reductions, so agreement is to
rounding, not bit for bit)."""
import numpy as np
import pytest

from amigo_b200 import ipm_driver
from amigo_b200.problems.cartpole import batch_config

pytestmark = pytest.mark.gpu


def test_batch_matches_individual_solves():
    B = batch_config(k=6, seed=3, nmin=50, nmax=150)
    r = ipm_driver.solve_batch(B, "cuda:0")
    assert r["converged"].all()
    assert (r["kkt_error"] <= 1e-8).all()
    for k, m in enumerate(B.inst):
        prob = ipm_driver.CartPoleProblem(m, "cuda:0")
        one = ipm_driver.solve(ipm_driver.DeviceBackend(prob, m, "cuda:0"))
        assert one["converged"]
        assert r["iterations"][k] == one["iterations"], k
        assert abs(r["objective"][k] - one["objective"]) <= 1e-9 * abs(one["objective"])
        xk = r["x"][B.var_off[k]:B.var_off[k + 1]]
        npr = m.npr
        assert np.abs(xk[:npr] - one["x"][:npr]).max() <= 1e-7
        # the pole ends upright at the drawn final cart position
        assert abs(xk[5 * m.N + 1] - np.pi) <= 1e-6
        assert abs(xk[5 * m.N] - m.xf) <= 1e-6


def test_batch_of_one_equals_config_size():
    B = batch_config(k=1, seed=5, nmin=100, nmax=100)
    r = ipm_driver.solve_batch(B, "cuda:0")
    assert r["converged"].all() and r["kkt_error"][0] <= 1e-8


def test_batch_mixed_precision_matches_fp64():
    """FP32 fronts with FP64 refinement: every instance converges to the
    FP64 batch's optimum (1e-9 relative objective, KKT error <= 1e-8).  An
    attempt whose FP32 inertia is not the wanted one is refactored in FP64
    before the inertia correction decides (counted in inertia_fallbacks)."""
    B = batch_config(k=6, seed=3, nmin=50, nmax=150)
    r64 = ipm_driver.solve_batch(B, "cuda:0", rescue=False)
    r32 = ipm_driver.solve_batch(B, "cuda:0", precision="fp32", rescue=False)
    assert r64["converged"].all() and r32["converged"].all()
    assert (r32["kkt_error"] <= 1e-8).all()
    rel = np.abs(r32["objective"] - r64["objective"]) / np.abs(r64["objective"])
    assert rel.max() <= 1e-9, rel
    assert r32["inertia_fallbacks"] >= 0 and r32["fallbacks"] >= 0


def test_threaded_reference_resolves_equal_sequential():
    """Re-solves by optimizer.Optimizer on several host threads (one CUDA
    stream each) give the results of the same re-solves one after
    another, bit for bit."""
    B = batch_config(k=3, seed=9, nmin=50, nmax=120)
    seq = ipm_driver._solve_reference_algorithm_many(B.inst, "cuda:0", 1)
    par = ipm_driver._solve_reference_algorithm_many(B.inst, "cuda:0", 3)
    for a, b in zip(seq, par):
        assert a["converged"] and b["converged"]
        assert a["iterations"] == b["iterations"]
        assert a["objective"] == b["objective"]
        assert np.array_equal(a["x"], b["x"])
