"""Host logic of the serving loop (serve.Server.run) on CPU, with a stand-in
for the batched engine: admission by slot count and memory budget at
iteration boundaries, retirement with latencies, re-solves of unconverged
requests on worker threads (rescue), and the over-budget error."""
import time

import pytest

from amigo_b200 import serve


class FakeEngine:
    """Admits (id, model) pairs; every instance retires after `iters` steps,
    converged when its id is even."""
    max_live = 0
    max_bytes = 0.0

    def __init__(self, device, options=None, precision="fp64", iters=3):
        self.live_ids = {}
        self.iters = iters
        self.rebuilds = 0
        self.rebuild_s = 0.0
        self.fallbacks = 0
        self.admitted = []
        self.bytes = {}

    def admit(self, items):
        for rid, m in items:
            self.live_ids[rid] = 0
            self.bytes[rid] = serve.workspace_bytes(m)
            self.admitted.append(rid)
        FakeEngine.max_live = max(FakeEngine.max_live, len(self.live_ids))
        FakeEngine.max_bytes = max(FakeEngine.max_bytes,
                                   sum(self.bytes[r] for r in self.live_ids))

    def live(self):
        return len(self.live_ids)

    def dead_fraction(self):
        return 0.0

    def step(self, rebuild=False):
        if rebuild:
            self.rebuilds += 1
        out = []
        for rid in list(self.live_ids):
            self.live_ids[rid] += 1
            if self.live_ids[rid] >= self.iters:
                del self.live_ids[rid]
                out.append(dict(id=rid, converged=rid % 2 == 0, iterations=self.iters,
                                t_done=time.perf_counter()))
        return out


@pytest.fixture
def fake(monkeypatch):
    FakeEngine.max_live = 0
    FakeEngine.max_bytes = 0.0
    monkeypatch.setattr(serve, "BatchEngine", FakeEngine)


def stream(n):
    return serve.make_stream(n, rate=2000.0, seed=1, nmin=20, nmax=30)


def test_admission_and_retirement(fake):
    reqs = stream(12)
    srv = serve.Server("cpu", max_batch=4, admit_min=1, max_wait_s=0.0)
    res, summ = srv.run(reqs, time_limit=60)
    assert summ["completed"] == 12 and summ["rescued"] == 0
    assert summ["converged"] == 6
    assert FakeEngine.max_live <= 4
    assert sorted(srv.engine.admitted) == [q.id for q in reqs]
    for q in reqs:
        assert res[q.id]["latency_s"] >= 0.0
        assert res[q.id]["converged"] == (q.id % 2 == 0)


def test_memory_budget_bounds_the_batch(fake):
    reqs = stream(8)
    one = max(serve.workspace_bytes(q.model()) for q in reqs)
    srv = serve.Server("cpu", mem_budget=2.5 * one, max_batch=8, admit_min=1,
                       max_wait_s=0.0)
    _, summ = srv.run(reqs, time_limit=60)
    assert summ["completed"] == 8
    assert 0.0 < FakeEngine.max_bytes <= 2.5 * one
    assert FakeEngine.max_live < 8


def test_over_budget_request_is_an_error(fake):
    reqs = stream(2)
    srv = serve.Server("cpu", mem_budget=1.0, admit_min=1, max_wait_s=0.0)
    with pytest.raises(ValueError, match="memory budget"):
        srv.run(reqs, time_limit=60)


def test_rescue_resolves_unconverged_requests(fake, monkeypatch):
    def resolve(self, m):
        time.sleep(0.01)
        return dict(converged=True, iterations=7, t_done=time.perf_counter(),
                    model_N=m.N)

    monkeypatch.setattr(serve.Server, "_resolve", resolve)
    reqs = stream(10)
    srv = serve.Server("cpu", max_batch=3, admit_min=1, max_wait_s=0.0,
                       rescue=True, rescue_workers=2)
    res, summ = srv.run(reqs, time_limit=60)
    assert summ["completed"] == 10 and summ["converged"] == 10
    assert summ["rescued"] == 5
    for q in reqs:
        r = res[q.id]
        assert r.get("rescued", False) == (q.id % 2 == 1)
        if r.get("rescued"):
            assert r["model_N"] == q.N and r["iterations"] == 7
        assert r["latency_s"] >= 0.0
