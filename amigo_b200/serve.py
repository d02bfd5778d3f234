"""Serving loop: a stream of interior-point solve requests with arrival
times, served by continuous batching on `batch_engine.BatchEngine`.

Requests that arrive while others are on the GPU are admitted at the next
iteration boundary as slots and device memory free up; converged (or
iteration-limited) problems retire at iteration boundaries and return their
results.  Admission is bounded by a device-memory budget computed from each
problem's symbolic analysis (front sizes of its multifrontal factorization,
cached per pattern) and by a slot count.  A rebuild of the batch (needed to
admit) is taken when enough requests wait, when the GPU would otherwise
idle, or when the oldest waiting request has waited `max_wait_s`; half a
layout of retired problems is compacted away too.

Requests here are cart-pole trajectory problems (problems/cartpole.py):
N ~ U{nmin..nmax} intervals, pole mass ~ U(0.1, 0.5), final cart position
~ U(-1, 1), from the seed.
"""
import time
from dataclasses import dataclass

import numpy as np
import torch

from .batch_engine import BatchEngine


@dataclass
class Request:
    id: int
    arrival: float       # seconds after the stream starts
    N: int
    m_pole: float
    xf: float
    seed: int

    def model(self):
        from .problems.cartpole import CartPole
        return CartPole(N=self.N, m_pole=self.m_pole, xf=self.xf, seed=self.seed)


def make_stream(n_requests, rate, seed=0, nmin=50, nmax=400):
    """Poisson arrivals at `rate` per second, parameters from the seed."""
    r = np.random.RandomState(seed)
    t = np.cumsum(r.exponential(1.0 / rate, n_requests))
    Ns = r.randint(nmin, nmax + 1, n_requests)
    ms = r.uniform(0.1, 0.5, n_requests)
    xfs = r.uniform(-1.0, 1.0, n_requests)
    return [Request(i, float(t[i]), int(Ns[i]), float(ms[i]), float(xfs[i]),
                    seed + 1 + i) for i in range(n_requests)]


_EST = {}


def workspace_bytes(model, delay_growth=2.0, precision=64):
    """Device bytes one problem needs: the factorization's workspace from its
    symbolic analysis (linalg.mem_estimate, the library's
    ab_ldl_mem_estimate: front pool with room for delayed pivots, integer
    pools, plan, solve vectors), plus the CSR values and ~24 n-vectors of
    iterate and work space.  Cached per pattern (n, nnz, precision)."""
    from .linalg import mem_estimate
    key = (model.n, model.nnz, precision)
    if key not in _EST:
        ws = mem_estimate(model.n, model.rowp, model.cols, precision=precision,
                          delay_growth=delay_growth)
        _EST[key] = ws + 20.0 * model.nnz + 8.0 * 24 * model.n
    return _EST[key]


class Server:
    def __init__(self, device="cuda", mem_budget=150e9, max_batch=512,
                 admit_min=64, max_wait_s=0.5, options=None, precision="fp64"):
        self.device = torch.device(device)
        self.mem_budget = mem_budget
        self.max_batch = max_batch
        self.admit_min = admit_min
        self.max_wait_s = max_wait_s
        self.engine = BatchEngine(self.device, options, precision)

    def run(self, requests, time_limit=None):
        """Serve `requests` in real time (arrival times relative to the
        call).  Returns (results by request id, summary)."""
        eng = self.engine
        pending = sorted(requests, key=lambda q: q.arrival)
        req = {q.id: q for q in pending}
        arrived = []                 # (request, model, bytes), arrival order
        resident = {}                # id -> bytes
        results = {}
        steps = 0
        t0 = time.perf_counter()
        while pending or arrived or eng.live():
            now = time.perf_counter() - t0
            if time_limit is not None and now > time_limit:
                break
            while pending and pending[0].arrival <= now:
                q = pending.pop(0)
                m = q.model()
                arrived.append((q, m, workspace_bytes(m)))
            if not arrived and not eng.live():
                # idle until the next arrival
                time.sleep(max(0.0, min(0.05, pending[0].arrival - now)))
                continue
            used = sum(resident.values())
            free = self.max_batch - eng.live()
            take = []
            while (arrived and len(take) < free
                   and used + arrived[0][2] <= self.mem_budget):
                q, m, b = arrived.pop(0)
                take.append((q, m, b))
                used += b
            if take:
                ready = (len(take) >= self.admit_min or eng.live() == 0
                         or now - take[0][0].arrival >= self.max_wait_s
                         or not pending)
                if not ready:
                    arrived = take + arrived    # keep them waiting, in order
                    take = []
            if take:
                eng.admit([(q.id, m) for q, m, _ in take])
                for q, _, b in take:
                    resident[q.id] = b
            if not eng.live():
                if arrived and not take:
                    raise ValueError("request %d needs %.3g bytes, more than the "
                                     "memory budget" % (arrived[0][0].id, arrived[0][2]))
                continue
            # admissions, or compaction once half the layout has retired
            for r in eng.step(rebuild=bool(take) or eng.dead_fraction() >= 0.5):
                q = req[r["id"]]
                r["latency_s"] = r["t_done"] - t0 - q.arrival
                results[r["id"]] = r
                resident.pop(r["id"], None)
            steps += 1
        wall = time.perf_counter() - t0
        lat = (np.array([r["latency_s"] for r in results.values()])
               if results else np.zeros(1))
        conv = sum(1 for r in results.values() if r["converged"])
        summary = dict(requests=len(requests), completed=len(results),
                       converged=conv, wall_s=wall,
                       solves_per_s=conv / wall if wall > 0 else 0.0,
                       p50_ms=1e3 * float(np.percentile(lat, 50)),
                       p95_ms=1e3 * float(np.percentile(lat, 95)),
                       p99_ms=1e3 * float(np.percentile(lat, 99)),
                       iterations=steps, rebuilds=eng.rebuilds,
                       rebuild_s=eng.rebuild_s,
                       fp64_fallbacks=eng.fallbacks)
        return results, summary
