"""Continuous batching (serve.Server on batch_engine.BatchEngine): requests
arriving while others are being solved are admitted at iteration
boundaries.  Bar: every request's result in the mix equals its result when
solved alone -- same iteration count, objective and optimum to 1e-12
relative (no computation mixes instances) -- under a small slot count and a
memory budget that force several admissions and retirements mid-solve."""
import numpy as np
import pytest

from amigo_b200 import ipm_driver, serve
from amigo_b200.problems.cartpole import CartPoleBatch

pytestmark = pytest.mark.gpu


def test_results_same_alone_and_in_the_mix():
    reqs = serve.make_stream(10, rate=40.0, seed=7, nmin=50, nmax=120)
    big = max(serve.workspace_bytes(q.model()) for q in reqs)
    srv = serve.Server("cuda:0", mem_budget=6 * big, max_batch=5, admit_min=2,
                       max_wait_s=0.05)
    res, summ = srv.run(reqs, time_limit=600)
    assert summ["completed"] == len(reqs)
    assert summ["rebuilds"] >= 3
    for q in reqs:
        r = res[q.id]
        alone = ipm_driver.solve_batch(CartPoleBatch([q.model()]), "cuda:0")
        assert r["converged"] == bool(alone["converged"][0])
        assert r["iterations"] == int(alone["iterations"][0])
        ref = alone["objective"][0]
        assert abs(r["objective"] - ref) <= 1e-12 * max(1.0, abs(ref))
        assert np.abs(r["x"] - alone["x"]).max() <= 1e-12 * max(1.0, np.abs(alone["x"]).max())
        assert r["latency_s"] > 0.0


def test_unconverged_requests_resolved_when_asked():
    """rescue=True: a request the batched driver leaves unconverged (here
    forced by a 5-iteration limit) is solved again by optimizer.Optimizer on
    a worker thread while the batch keeps stepping, and converges."""
    reqs = serve.make_stream(4, rate=100.0, seed=3, nmin=50, nmax=80)
    srv = serve.Server("cuda:0", max_batch=4, admit_min=1, max_wait_s=0.01,
                       options={"max_iter": 5}, rescue=True, rescue_workers=2)
    res, summ = srv.run(reqs, time_limit=600)
    assert summ["completed"] == len(reqs) and summ["rescued"] == len(reqs)
    assert summ["converged"] == len(reqs)
    for q in reqs:
        r = res[q.id]
        assert r["rescued"] and r["converged"] and r["latency_s"] > 0.0
