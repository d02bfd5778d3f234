"""Whole interior-point solves of the reference's own Hock-Schittkowski test
problems (its examples/test_problems; components serialized by the
reference, tests/golden/ref_components.json) with equality constraints
only: each problem is one component instance, its derivatives the
generated evaluators of codegen.from_amigo (host build).  The reference's
own Optimizer (oracle/ref_optimizer.py: its driver, AmigoSolver and
SparseLDL over its C++ backend) and this package's optimizer.Optimizer run
on the same host numeric core; every iteration record (residual, barrier
parameter, step lengths, line-search trials, inertia perturbation, the KKT
error terms, objective) and the final iterate must be the same bits.
Inequality rows get a bounded slack each (c(x) - s = 0), the same problem
for both drivers.  CPU only; needs the reference sources."""
import json
import os
import types

import numpy as np
import pytest

from amigo_b200 import codegen as cg

FIX = os.path.join(os.path.dirname(__file__), "golden", "ref_components.json")
REF = os.environ.get("AMIGO_REF_ROOT", "/root/reference")
FIELDS = ("residual", "barrier_param", "alpha_x", "alpha_z", "line_iters",
          "inertia_delta", "inf_pr", "inf_du", "compl", "nlp_error", "objective")
needs_ref = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "amigo", "algorithm")),
                               reason="reference sources absent")

EQ_ONLY = ("HS6", "HS26", "HS39", "HS40", "HS53", "HS60", "HS77", "HS79", "HS99",
           "HS111", "HS119", "HS87")
WITH_INEQ = ("HS14", "HS29", "HS35", "HS44", "HS71", "HS76", "HS93", "HS100", "HS104",
             "HS106", "HS108", "HS109", "HS113", "HS114", "HS116", "HS117", "HS118",
             "Rosenbrock")


def problem(name):
    """The single-instance model of one test problem: inputs, one slack per
    inequality constraint entry (c(x) - s = 0 with s within the
    constraint's bounds), then one multiplier per constraint entry; a dense
    KKT block; bounds and start from the component's metadata (equality
    targets as the multipliers' lower bounds)."""
    comps = json.load(open(FIX))["components"]
    c = next(c for c in comps if c["cls"] == name)
    comp = cg.from_amigo(c["data"])
    ev = cg.host_evaluator(comp, "hs_" + name.lower())
    ni, nq, nd = comp.num_inputs, comp.num_vars, comp.num_data
    nc = nq - ni
    lo, hi = comp.input_bounds()
    x0 = np.zeros(ni)
    k = 0
    for nm in comp._inputs:
        v = np.asarray(comp._inputs.meta[nm]["value"], float)
        n = int(np.prod(comp._inputs.shapes[nm])) if comp._inputs.shapes[nm] else 1
        x0[k:k + n] = np.broadcast_to(v, (n,))
        k += n
    clo, chi = [], []
    for nm in comp._cons:
        n = int(np.prod(comp._cons.shapes[nm])) if comp._cons.shapes[nm] else 1
        m_ = comp._cons.meta[nm]
        clo += list(np.broadcast_to(np.asarray(m_["lower"], float), (n,)))
        chi += list(np.broadcast_to(np.asarray(m_["upper"], float), (n,)))
    clo, chi = np.array(clo), np.array(chi)
    ineq = np.nonzero(clo < chi)[0]            # constraint rows with a slack
    ns = len(ineq)
    n = ni + ns + nc
    S, M = slice(ni, ni + ns), slice(ni + ns, n)
    tgt = np.where(clo < chi, 0.0, clo)
    m = types.SimpleNamespace(
        n=n, mult=np.arange(n) >= ni + ns,
        lower=np.concatenate([lo, clo[ineq], tgt]),
        upper=np.concatenate([hi, chi[ineq], np.full(nc, np.inf)]),
        x0=np.concatenate([x0, np.zeros(ns + nc)]),
        rowp=np.arange(0, n * n + 1, n, dtype=np.int32),
        cols=np.tile(np.arange(n, dtype=np.int32), n),
        diag_pos=np.arange(n) * (n + 1))
    d = np.zeros(max(nd, 1))
    sel = np.r_[0:ni, ni + ns:n]               # the component's own variables

    def evx(x, a):
        return ev(x[sel], d, a)

    def grad(x, a):
        gq, _, _ = evx(x, a)
        g = np.zeros(n)
        g[:ni] = gq[:ni]
        g[M] = gq[ni:]
        g[M][ineq] -= x[S]                     # c - s on the slack rows
        g[S] = -x[M][ineq]                     # d/ds of -lam s
        return g

    def hess(x, a):
        _, Hq, _ = evx(x, a)
        H = np.zeros((n, n))
        H[np.ix_(sel, sel)] = Hq
        rows = ni + ns + ineq
        H[np.arange(ni, ni + ns), rows] = -1.0
        H[rows, np.arange(ni, ni + ns)] = -1.0
        return H.ravel()

    def lag(x, a):
        gq, _, f = evx(x, a)
        cval = gq[ni:].copy()
        cval[ineq] -= x[S]
        return a * f + x[M] @ cval

    obj = lambda x: evx(x, 1.0)[2]
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
@pytest.mark.parametrize("name", EQ_ONLY + WITH_INEQ)
def test_hs_problem_matches_reference_optimizer(oracle_ref, name):
    from oracle import ref_optimizer as RO
    m, grad, hess, lag, obj = problem(name)
    want = RO.optimize(m, grad, hess, lag, obj)
    got = ours(m, grad, hess, lag)
    assert got["converged"] == want["converged"]
    assert len(got["iterations"]) == len(want["records"])
    for a, b in zip(got["iterations"], want["records"]):
        for k in FIELDS:
            if b.get(k) is None or isinstance(b.get(k), str):
                continue
            assert float(a[k]) == float(b[k]), (name, a["iteration"], k)
    assert np.array_equal(got["x"], want["x"])


def generated_model(name):
    """The same problem as a GeneratedModel: one instance of the imported
    component (inputs then multipliers) and codegen.with_slacks for the
    inequality rows (slacks appended)."""
    comps = json.load(open(FIX))["components"]
    c = next(c for c in comps if c["cls"] == name)
    comp = cg.from_amigo(c["data"])
    ni, nq = comp.num_inputs, comp.num_vars
    lo, hi = comp.input_bounds()
    clo, chi = [], []
    for nm in comp._cons:
        n = int(np.prod(comp._cons.shapes[nm])) if comp._cons.shapes[nm] else 1
        clo += list(np.broadcast_to(np.asarray(comp._cons.meta[nm]["lower"], float), (n,)))
        chi += list(np.broadcast_to(np.asarray(comp._cons.meta[nm]["upper"], float), (n,)))
    clo, chi = np.array(clo), np.array(chi)
    ineq = np.nonzero(clo < chi)[0]
    x0 = np.zeros(nq)
    x0[:ni] = problem(name)[0].x0[:ni]
    G = cg.with_slacks(nq, [cg.Group(comp, np.arange(nq)[None, :], name=name)],
                       np.arange(nq) >= ni, np.concatenate([lo, clo]),
                       np.concatenate([hi, np.full(nq - ni, np.inf)]),
                       ni + ineq, clo[ineq], chi[ineq], x0=x0)
    return G, ni, ineq


@pytest.mark.parametrize("name", ("HS14", "HS71", "HS100", "Rosenbrock"))
def test_with_slacks_matches_hand_augmented(name):
    """with_slacks gives the derivatives of the hand-built slack form
    (variables permuted: the model appends its slacks)."""
    m, grad, hess, _, _ = problem(name)
    G, ni, ineq = generated_model(name)
    ns, n = len(ineq), m.n
    # hand form: inputs, slacks, multipliers; model: inputs, multipliers, slacks
    perm = np.r_[0:ni, ni + ns:n, ni:ni + ns]
    assert G.n == n and np.array_equal(G.mult, m.mult[perm])
    assert np.array_equal(G.lower, m.lower[perm]) and np.array_equal(G.upper, m.upper[perm])
    x = 0.3 + 0.5 * np.random.RandomState(1).rand(n)
    g, vals = G.host_derivatives(x[perm], 0.7)
    assert np.allclose(g, grad(x, 0.7)[perm], rtol=1e-14, atol=1e-14)
    Hd = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(G.rowp))
    Hd[rows, G.cols] = vals
    assert np.allclose(Hd, hess(x, 0.7).reshape(n, n)[np.ix_(perm, perm)],
                       rtol=1e-14, atol=1e-14)
    assert np.array_equal(G.slack_indices, np.arange(n - ns, n))


@needs_ref
@pytest.mark.parametrize("name", ("HS71", "HS100", "HS118"))
def test_generated_model_solves_match(oracle_ref, name):
    """Both drivers on the GeneratedModel (sparse KKT pattern) agree bit
    for bit, and converge to the dense form's objective."""
    from oracle import ref_optimizer as RO
    G, ni, ineq = generated_model(name)
    grad = lambda x, a: G.host_derivatives(x, a)[0]
    hess = lambda x, a: G.host_derivatives(x, a)[1]
    lag = lambda x, a: G.host_lagrangian(x, a)
    obj = lambda x: G.host_lagrangian(x * ~G.mult, 1.0)
    m = types.SimpleNamespace(n=G.n, mult=G.mult, lower=G.lower, upper=G.upper, x0=G.x0,
                              rowp=G.rowp, cols=G.cols, diag_pos=G.diag_pos)
    want = RO.optimize(m, grad, hess, lag, obj)
    got = ours(m, grad, hess, lag)
    assert got["converged"] and want["converged"]
    assert len(got["iterations"]) == len(want["records"])
    for a, b in zip(got["iterations"], want["records"]):
        for k in FIELDS:
            if b.get(k) is None or isinstance(b.get(k), str):
                continue
            assert float(a[k]) == float(b[k]), (name, a["iteration"], k)
    dense = problem(name)
    ref_dense = RO.optimize(*dense)
    assert abs(obj(got["x"]) - ref_dense["objective"]) <= 1e-7 * max(1.0, abs(ref_dense["objective"]))


@needs_ref
def test_sellar_multi_component_model(oracle_ref):
    """The reference's Sellar example: its five components (imported from
    their reference serialization) share the inputs of the same name, as
    its Model.link_by_name links them; its bounds, start and optimizer
    options.  Both drivers run the generated model on the same host core
    and agree bit for bit."""
    from oracle import ref_optimizer as RO
    comps = {c["cls"]: c for c in json.load(open(FIX))["components"]
             if c["source"].endswith("sellar.py")}
    names = ["x", "z1", "z2", "y1", "y2"]
    groups, ncon = [], 0
    for cls in ("Disp1", "Disp2", "Objective", "Con1", "Con2"):
        comp = cg.from_amigo(comps[cls]["data"])
        idx = [names.index(k) for k in comp._inputs]
        idx += list(range(len(names) + ncon, len(names) + ncon + comp.num_constraints))
        ncon += comp.num_constraints
        groups.append(cg.Group(comp, np.array([idx]), name=cls))
    n = len(names) + ncon
    mult = np.arange(n) >= len(names)
    # the example's vectors: lower from a zero vector with x, y1, z1 set to
    # -inf; upper +inf on the inputs; constraint targets 0
    lower = np.zeros(n)
    lower[[0, 1, 3]] = -np.inf
    upper = np.zeros(n)
    upper[:len(names)] = np.inf
    x0 = np.zeros(n)
    x0[[1, 2, 3, 4]] = 1.0
    G = cg.GeneratedModel(n, groups, mult, lower, upper, x0=x0)
    grad = lambda x, a: G.host_derivatives(x, a)[0]
    hess = lambda x, a: G.host_derivatives(x, a)[1]
    lag = lambda x, a: G.host_lagrangian(x, a)
    obj = lambda x: G.host_lagrangian(x * ~G.mult, 1.0)
    m = types.SimpleNamespace(n=n, mult=mult, lower=lower, upper=upper, x0=x0,
                              rowp=G.rowp, cols=G.cols, diag_pos=G.diag_pos)
    opts = {"initial_barrier_param": 0.1, "max_line_search_iterations": 1,
            "max_iterations": 500, "init_affine_step_multipliers": False}
    want = RO.optimize(m, grad, hess, lag, obj, options=opts)

    from amigo_b200.optimizer import Optimizer
    alg = RO.install()
    P = RO.HostProblem(m, grad, hess, lag)
    opt = Optimizer(P, RO.HostVector(arr=x0.copy()), RO.HostVector(arr=lower.copy()),
                    RO.HostVector(arr=upper.copy()), alg.solvers.AmigoSolver(P),
                    backend_class=RO.InteriorPointOptimizer)
    got = opt.optimize(dict(opts))
    assert got["converged"] == want["converged"]
    assert len(got["iterations"]) == len(want["records"])
    for a, b in zip(got["iterations"], want["records"]):
        for k in FIELDS:
            if b.get(k) is None or isinstance(b.get(k), str):
                continue
            assert float(a[k]) == float(b[k]), (a["iteration"], k)
    assert np.array_equal(np.array(opt.vars.get_solution().arr), want["x"])


@needs_ref
def test_every_amigo_option_name_is_accepted():
    """Every option of amigo's get_default_options is known here: the
    restated ones take any value, the others their default (the default
    algorithm) and raise NotImplementedError otherwise; unknown names are a
    ValueError, as in amigo."""
    import importlib
    from amigo_b200 import optimizer as O
    from oracle import ref_optimizer as RO
    RO.install()
    ref = importlib.import_module("amigo.algorithm.default_options").get_default_options()
    assert set(ref) == set(O.DEFAULT_OPTIONS) | set(O.DEFAULT_ALGORITHM_OPTIONS)
    for k, v in O.DEFAULT_ALGORITHM_OPTIONS.items():
        assert ref[k] == v, k
    for k, v in O.DEFAULT_OPTIONS.items():
        assert ref[k] == v, k
    m, grad, hess, lag, _ = problem("HS6")
    alg = RO.install()
    P = RO.HostProblem(m, grad, hess, lag)

    def run(opts):
        opt = O.Optimizer(P, RO.HostVector(arr=m.x0.copy()), RO.HostVector(arr=m.lower.copy()),
                          RO.HostVector(arr=m.upper.copy()), alg.solvers.AmigoSolver(P),
                          backend_class=RO.InteriorPointOptimizer)
        return opt.optimize(opts)
    assert run(dict(O.DEFAULT_ALGORITHM_OPTIONS, verbose_barrier=True))["converged"]
    with pytest.raises(NotImplementedError, match="barrier_strategy"):
        run({"barrier_strategy": "quality_function"})
    with pytest.raises(ValueError, match="Unrecognized option"):
        run({"no_such_option": 1})


@needs_ref
def test_reference_cart_pole_model(oracle_ref):
    """The reference's cart-pole trajectory example (its create_cart_model,
    100 steps): its components imported from their reference serialization
    and laid out as its links lay them out -- cart instances k = 0..100,
    trapezoid instance i*100 + k joining state i of carts k and k+1, the
    objective joining the controls of carts k and k+1, initial and final
    conditions on carts 0 and 100 -- with its start values and data.  Both
    drivers agree bit for bit on the generated model."""
    from oracle import ref_optimizer as RO
    comps = {c["cls"]: c for c in json.load(open(FIX))["components"]
             if c["source"].endswith("cart_pole.py")}
    N = 100
    cart = cg.from_amigo(comps["CartComponent"]["data"])
    trap = cg.from_amigo(comps["TrapezoidRule"]["data"])
    objc = cg.from_amigo(comps["Objective"]["data"])
    ic = cg.from_amigo(comps["InitialConditions"]["data"])
    fc = cg.from_amigo(comps["FinalConditions"]["data"])
    nv = 9                                   # x, q[4], qdot[4] per cart
    X = lambda k: k * nv
    Q = lambda k, i: k * nv + 1 + i
    QD = lambda k, i: k * nv + 5 + i
    nxt = [nv * (N + 1)]

    def mults(count):
        a = np.arange(nxt[0], nxt[0] + count)
        nxt[0] += count
        return a
    cart_idx = np.array([[X(k)] + [Q(k, i) for i in range(4)] + [QD(k, i) for i in range(4)]
                         + list(mults(4)) for k in range(N + 1)])
    trap_idx = np.array([[Q(k, i), Q(k + 1, i), QD(k, i), QD(k + 1, i)] + list(mults(1))
                         for i in range(4) for k in range(N)])
    obj_idx = np.array([[X(k), X(k + 1)] for k in range(N)])
    ic_idx = np.array([[Q(0, i) for i in range(4)] + list(mults(4))])
    fc_idx = np.array([[Q(N, i) for i in range(4)] + list(mults(4))])
    n = nxt[0]
    data = np.tile([0.5, 1.0, 0.3], (N + 1, 1))       # L, m1, m2
    groups = [cg.Group(cart, cart_idx, data, name="cart"), cg.Group(trap, trap_idx, name="trap"),
              cg.Group(objc, obj_idx, name="obj"), cg.Group(ic, ic_idx, name="ic"),
              cg.Group(fc, fc_idx, name="fc")]
    mult = np.arange(n) >= nv * (N + 1)
    lower = np.where(mult, 0.0, -np.inf)
    upper = np.where(mult, 0.0, np.inf)
    lower[[X(k) for k in range(N + 1)]] = -50.0
    upper[[X(k) for k in range(N + 1)]] = 50.0
    upper[mult] = np.inf
    x0 = np.zeros(n)
    x0[[Q(k, 0) for k in range(N + 1)]] = np.linspace(0.0, 2.0, N + 1)
    x0[[Q(k, 1) for k in range(N + 1)]] = np.linspace(0.0, np.pi, N + 1)
    x0[[Q(k, 2) for k in range(N + 1)]] = 1.0
    x0[[Q(k, 3) for k in range(N + 1)]] = 1.0
    G = cg.GeneratedModel(n, groups, mult, lower, upper, x0=x0)
    cache = {}

    def deriv(x, a):
        key = (x.tobytes(), a)
        if key not in cache:
            cache.clear()
            cache[key] = G.host_derivatives(x, a)
        return cache[key]
    grad = lambda x, a: deriv(x, a)[0]
    hess = lambda x, a: deriv(x, a)[1]
    lag = lambda x, a: G.host_lagrangian(x, a)
    obj = lambda x: G.host_lagrangian(x * ~G.mult, 1.0)
    m = types.SimpleNamespace(n=n, mult=mult, lower=lower, upper=upper, x0=x0,
                              rowp=G.rowp, cols=G.cols, diag_pos=G.diag_pos)
    want = RO.optimize(m, grad, hess, lag, obj)
    got = ours(m, grad, hess, lag)
    assert want["converged"] and got["converged"]
    assert len(got["iterations"]) == len(want["records"])
    for a, b in zip(got["iterations"], want["records"]):
        for k in FIELDS:
            if b.get(k) is None or isinstance(b.get(k), str):
                continue
            assert float(a[k]) == float(b[k]), (a["iteration"], k)
    assert np.array_equal(got["x"], want["x"])
    # the swing-up reaches its final conditions
    xs = got["x"]
    assert abs(xs[Q(N, 0)] - 2.0) < 1e-6 and abs(xs[Q(N, 1)] - np.pi) < 1e-6
