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
layout of retired problems is compacted away too.  With `rescue`, a
request the batched driver leaves unconverged is solved again by
optimizer.Optimizer (amigo's default algorithm) on a pool of host threads,
each with its own CUDA stream, while the batch keeps stepping; its result
is that re-solve's, as in ipm_driver.solve_batch.  It is off by default:
the re-solve threads share the interpreter with the batch loop and slowed
it (600 cart-pole requests: all converged at 27 solves/s with it, 582 of
600 at 42 solves/s without).

Requests here are cart-pole trajectory problems (problems/cartpole.py):
N ~ U{nmin..nmax} intervals, pole mass ~ U(0.1, 0.5), final cart position
~ U(-1, 1), from the seed.
"""
import threading
import time
from concurrent.futures import ThreadPoolExecutor
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
                 admit_min=64, max_wait_s=0.5, options=None, precision="fp64",
                 rescue=False, rescue_workers=4):
        self.device = torch.device(device)
        self.mem_budget = mem_budget
        self.max_batch = max_batch
        self.admit_min = admit_min
        self.max_wait_s = max_wait_s
        self.engine = BatchEngine(self.device, options, precision)
        self.rescue = rescue
        self.rescue_workers = rescue_workers
        self._local = threading.local()

    def _resolve(self, m):
        """optimizer.Optimizer on `m`, on this worker thread's own stream."""
        from .ipm_driver import _solve_reference_algorithm
        s = getattr(self._local, "stream", None)
        if s is None:
            s = self._local.stream = torch.cuda.Stream(device=self.device)
        with torch.cuda.stream(s):
            r = _solve_reference_algorithm(m, self.device)
            s.synchronize()
        r["t_done"] = time.perf_counter()
        return r

    def run(self, requests, time_limit=None):
        """Serve `requests` in real time (arrival times relative to the
        call).  Returns (results by request id, summary)."""
        eng = self.engine
        pending = sorted(requests, key=lambda q: q.arrival)
        req = {q.id: q for q in pending}
        arrived = []                 # (request, model, bytes), arrival order
        resident = {}                # id -> bytes
        models = {}                  # id -> model, while in the batch
        resolving = {}               # id -> future of its re-solve
        results = {}
        steps = 0
        pool = (ThreadPoolExecutor(max_workers=self.rescue_workers)
                if self.rescue else None)
        if pool is not None and self.device.type == "cuda":
            torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()

        def collect():
            for rid in [i for i, fu in resolving.items() if fu.done()]:
                r = resolving.pop(rid).result()
                r["id"] = rid
                r["rescued"] = True
                r["latency_s"] = r["t_done"] - t0 - req[rid].arrival
                results[rid] = r

        while pending or arrived or eng.live() or resolving:
            collect()
            now = time.perf_counter() - t0
            if time_limit is not None and now > time_limit:
                break
            while pending and pending[0].arrival <= now:
                q = pending.pop(0)
                m = q.model()
                arrived.append((q, m, workspace_bytes(m)))
            if not arrived and not eng.live():
                # idle until the next arrival or re-solve
                wait = pending[0].arrival - now if pending else 0.005
                time.sleep(max(0.0, min(0.05, wait)))
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
                for q, m, b in take:
                    resident[q.id] = b
                    models[q.id] = m
            if not eng.live():
                if arrived and not take:
                    raise ValueError("request %d needs %.3g bytes, more than the "
                                     "memory budget" % (arrived[0][0].id, arrived[0][2]))
                continue
            # admissions, or compaction once half the layout has retired
            for r in eng.step(rebuild=bool(take) or eng.dead_fraction() >= 0.5):
                q = req[r["id"]]
                resident.pop(r["id"], None)
                m = models.pop(r["id"], None)
                if not r["converged"] and pool is not None:
                    resolving[r["id"]] = pool.submit(self._resolve, m)
                    continue
                r["latency_s"] = r["t_done"] - t0 - q.arrival
                results[r["id"]] = r
            steps += 1
        if pool is not None:
            pool.shutdown(wait=True, cancel_futures=True)
            collect()
        wall = time.perf_counter() - t0
        lat = (np.array([r["latency_s"] for r in results.values()])
               if results else np.zeros(1))
        conv = sum(1 for r in results.values() if r["converged"])
        summary = dict(requests=len(requests), completed=len(results),
                       converged=conv, wall_s=wall,
                       rescued=sum(1 for r in results.values() if r.get("rescued")),
                       solves_per_s=conv / wall if wall > 0 else 0.0,
                       p50_ms=1e3 * float(np.percentile(lat, 50)),
                       p95_ms=1e3 * float(np.percentile(lat, 95)),
                       p99_ms=1e3 * float(np.percentile(lat, 99)),
                       iterations=steps, rebuilds=eng.rebuilds,
                       rebuild_s=eng.rebuild_s,
                       fp64_fallbacks=eng.fallbacks)
        return results, summary
