"""Whole interior-point solves of the reference's own Hock-Schittkowski test
problems (its examples/test_problems; components serialized by the
reference, tests/golden/ref_components.json) with equality constraints
only: each problem is one component instance, its derivatives the
generated evaluators of codegen.from_amigo (host build).  The reference's
own Optimizer (oracle/ref_optimizer.py: its driver, AmigoSolver and
SparseLDL over its C++ backend) and this package's optimizer.Optimizer run
on the same host numeric core; they must converge alike, in the same
number of iterations (within one) and to the same objective (1e-8
relative).  CPU only; needs the reference sources."""
import json
import os
import types

import numpy as np
import pytest

from amigo_b200 import codegen as cg

FIX = os.path.join(os.path.dirname(__file__), "golden", "ref_components.json")
REF = os.environ.get("AMIGO_REF_ROOT", "/root/reference")
needs_ref = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "amigo", "algorithm")),
                               reason="reference sources absent")

EQ_ONLY = ("HS6", "HS26", "HS39", "HS40", "HS53", "HS60", "HS77", "HS79", "HS99",
           "HS111", "HS119", "HS87")


def problem(name):
    """The single-instance model of one test problem: inputs then one
    multiplier per constraint entry, a dense KKT block, bounds and start
    from the component's metadata (constraint targets as the multipliers'
    lower bounds)."""
    comps = json.load(open(FIX))["components"]
    c = next(c for c in comps if c["cls"] == name)
    comp = cg.from_amigo(c["data"])
    ev = cg.host_evaluator(comp, "hs_" + name.lower())
    ni, nq, nd = comp.num_inputs, comp.num_vars, comp.num_data
    lo, hi = comp.input_bounds()
    x0 = np.zeros(nq)
    k = 0
    for nm in comp._inputs:
        v = np.asarray(comp._inputs.meta[nm]["value"], float)
        n = int(np.prod(comp._inputs.shapes[nm])) if comp._inputs.shapes[nm] else 1
        x0[k:k + n] = np.broadcast_to(v, (n,))
        k += n
    tgt = []
    for nm in comp._cons:
        n = int(np.prod(comp._cons.shapes[nm])) if comp._cons.shapes[nm] else 1
        tgt += list(np.broadcast_to(np.asarray(comp._cons.meta[nm]["lower"], float), (n,)))
    m = types.SimpleNamespace(
        n=nq, mult=np.arange(nq) >= ni,
        lower=np.concatenate([lo, tgt]), upper=np.concatenate([hi, np.full(nq - ni, np.inf)]),
        x0=x0, rowp=np.arange(0, nq * nq + 1, nq, dtype=np.int32),
        cols=np.tile(np.arange(nq, dtype=np.int32), nq),
        diag_pos=np.arange(nq) * (nq + 1))
    d = np.zeros(max(nd, 1))
    grad = lambda x, a: ev(x, d, a)[0]
    hess = lambda x, a: ev(x, d, a)[1].ravel()

    def lag(x, a):
        g, _, f = ev(x, d, a)
        return a * f + x[ni:] @ g[ni:]
    obj = lambda x: ev(x, d, 1.0)[2]
    return m, grad, hess, lag, obj


def ours(m, grad, hess, lag):
    from amigo_b200.optimizer import Optimizer
    from oracle import ref_optimizer as RO
    alg = RO.install()
    P = RO.HostProblem(m, grad, hess, lag)
    solver = alg.solvers.AmigoSolver(P)
    x = RO.HostVector(arr=np.array(m.x0, dtype=np.float64))
    lo = RO.HostVector(arr=np.array(m.lower, dtype=np.float64))
    hi = RO.HostVector(arr=np.array(m.upper, dtype=np.float64))
    opt = Optimizer(P, x, lo, hi, solver, backend_class=RO.InteriorPointOptimizer)
    r = opt.optimize()
    r["x"] = np.array(opt.vars.get_solution().arr, dtype=np.float64)
    return r


@needs_ref
@pytest.mark.parametrize("name", EQ_ONLY)
def test_hs_problem_matches_reference_optimizer(oracle_ref, name):
    from oracle import ref_optimizer as RO
    m, grad, hess, lag, obj = problem(name)
    want = RO.optimize(m, grad, hess, lag, obj)
    got = ours(m, grad, hess, lag)
    assert got["converged"] == want["converged"]
    assert abs((len(got["iterations"]) - 1) - want["iterations"]) <= 1
    if want["converged"]:
        f = obj(got["x"])
        assert abs(f - want["objective"]) <= 1e-8 * max(1.0, abs(want["objective"]))
