"""Components serialized by the reference's own front end, run through this
package's code generator (codegen.from_amigo).  The fixture
(tests/golden/ref_components.json, made by make_ref_components.py) holds
the component classes of the reference's examples -- the cart-pole
trajectory, Sellar, Rosenbrock and the Hock-Schittkowski test problems --
and one component of the fixture script that uses the expression functions
the examples leave out, as the reference serialized them, with the value of
each serialized Lagrangian at two sample points (oracle/expr_oracle.py on
the reference's tree).  The generated evaluators (host build of the device
source) must give that Lagrangian, its gradient by central differences of
the reference's tree (passive subexpressions held), and a symmetric Hessian
equal to the differences of the gradient (with passive subexpressions:
second differences of the tree)."""
import json
import os

import numpy as np
import pytest

from amigo_b200 import codegen as cg
from oracle import expr_oracle as X

FIX = os.path.join(os.path.dirname(__file__), "golden", "ref_components.json")


@pytest.fixture(scope="module")
def generated():
    comps = json.load(open(FIX))["components"]
    built = [cg.from_amigo(c["data"]) for c in comps]
    evs = cg.host_evaluators([("ref%d" % i, b) for i, b in enumerate(built)])
    return comps, built, evs


def test_fixture_covers_the_examples(generated):
    comps, _, _ = generated
    names = {(c["source"].split("/")[-1], c["cls"]) for c in comps}
    assert ("cart_pole.py", "CartComponent") in names
    assert ("sellar.py", "Objective") in names
    assert sum(1 for s, _ in names if s.startswith("hs")) >= 20
    assert len(comps) >= 30


def test_layout_matches_the_reference(generated):
    comps, built, _ = generated
    for c, b in zip(comps, built):
        assert b.num_vars == X.num_vars(c["data"]), c["cls"]
        assert b.num_data == X.num_data(c["data"]), c["cls"]


def second_differences(data, x, d, alpha, h=1e-4):
    """Lower triangle of the Hessian of the reference tree's Lagrangian by
    second differences, passive subexpressions held at x."""
    n = len(x)
    H = np.zeros((n, n))
    L = lambda y: X.lagrangian(data, y, d, alpha, x_frozen=x)
    for i in range(n):
        for j in range(i + 1):
            ei = np.zeros(n)
            ej = np.zeros(n)
            ei[i] = h
            ej[j] = h
            H[i, j] = H[j, i] = (L(x + ei + ej) - L(x + ei - ej) - L(x - ei + ej)
                                 + L(x - ei - ej)) / (4 * h * h)
    return H


def test_lagrangian_gradient_hessian(generated):
    comps, built, evs = generated
    for c, b, ev in zip(comps, built, evs):
        data, ni = c["data"], b.num_inputs
        passive = "passive" in json.dumps(data)
        for p in c["points"]:
            x, d, alpha = np.array(p["x"]), np.array(p["d"]), p["alpha"]
            g, H, obj = ev(x, d, alpha)
            L = alpha * obj + x[ni:] @ g[ni:]
            Lref = p["lagrangian"]
            assert X.lagrangian(data, x, d, alpha) == Lref
            scale = max(1.0, abs(Lref))
            assert abs(L - Lref) <= 1e-12 * scale, (c["cls"], L, Lref)
            h = 1e-6
            gsc = max(scale, np.abs(g).max())
            for i in range(len(x)):
                e = np.zeros(len(x))
                e[i] = h
                fd = (X.lagrangian(data, x + e, d, alpha, x_frozen=x) -
                      X.lagrangian(data, x - e, d, alpha, x_frozen=x)) / (2 * h)
                assert abs(fd - g[i]) <= 1e-6 * gsc, (c["cls"], i, fd, g[i])
                if not passive:
                    gp, _, _ = ev(x + e, d, alpha)
                    gm, _, _ = ev(x - e, d, alpha)
                    col = (gp - gm) / (2 * h)
                    hsc = max(gsc, np.abs(H).max())
                    assert np.abs(col - H[:, i]).max() <= 1e-6 * hsc, (c["cls"], i)
            if passive:
                # the generated gradient moves with the passive values, so
                # the Hessian is checked against the tree directly
                Hd = second_differences(data, x, d, alpha)
                assert np.abs(Hd - H).max() <= 1e-5 * max(1.0, np.abs(H).max()), c["cls"]
            assert np.array_equal(H, H.T), c["cls"]


def test_json_text_and_bounds(generated):
    comps, built, _ = generated
    c = next(c for c in comps if c["cls"] == "CartComponent")
    b = cg.from_amigo(json.dumps(c["data"]))
    lo, hi = b.input_bounds()
    # the control x in [-50, 50]; q and qdot unbounded (amigo's defaults)
    assert lo[0] == -50.0 and hi[0] == 50.0
    assert np.all(np.isinf(lo[1:])) and np.all(np.isinf(hi[1:]))
    assert b.num_constraints == 4


def test_every_expression_function(generated):
    """The component the fixture script defines with the reference's API
    covers atan2, min2, max2, asinh, acosh, atanh and passive."""
    comps, _, _ = generated
    c = next(c for c in comps if c["cls"] == "AllFunctions")
    text = json.dumps(c["data"])
    for op in ("atan2", "min2", "max2", "asinh", "acosh", "atanh", "passive", "fabs"):
        assert '"%s"' % op in text, op


def test_rejected_nodes():
    base = {"name": "T", "args": [{}], "constants": {}, "data": {}, "outputs": {},
            "objective": {}, "lagrangian": {},
            "inputs": {"a": {"meta": {"shape": None}, "expr": ["var", "a", None, "float", True]}}}
    for tree, what in ((["binary", "hypot", ["var", "a", None, "float", True],
                         ["const", None, 1.0, "float"]], "hypot"),
                       (["unary", "erf", ["var", "a", None, "float", True]], "erf"),
                       (["lambda", ["var", "a", None, "float", True]], "lambda")):
        d = dict(base, constraints={"c": {"meta": {"shape": None},
                                          "expr": {"expr": {"0": {"expr": tree}}}}})
        with pytest.raises(ValueError, match=what):
            cg.from_amigo(d).build()
    with pytest.raises(ValueError, match="argument sets"):
        cg.from_amigo(dict(base, args=[{}, {}], constraints={}))


def test_device_module_compiles(generated):
    """The same generated source, built for sm_100a (nvcc cross-compiles
    without a GPU)."""
    import shutil
    from amigo_b200.codegen import emit
    from amigo_b200.codegen.model import compile_module
    if not (shutil.which("nvcc") or os.path.exists("/usr/local/cuda/bin/nvcc")):
        pytest.skip("nvcc not available")
    _, built, _ = generated
    src = emit.module_source([("ref%d" % i, b) for i, b in enumerate(built)])
    assert os.path.exists(compile_module(src, host=False))


def test_declarations_checked_like_amigo():
    """The declaration checks of amigo's Meta (amigo/meta.py): reserved
    double-underscore names, lower > upper, an input value outside its
    bounds, unknown options and misshaped values are ValueErrors; unset
    values take amigo's defaults."""
    bad = [lambda c: c.add_input("bad__name"),
           lambda c: c.add_input("x", lower=10.0, upper=1.0),
           lambda c: c.add_input("x", value=5.0, lower=0.0, upper=4.0),
           lambda c: c.add_input("x", unknown_kwarg=42),
           lambda c: c.add_input("x", shape=(3,), value=[1.0, 2.0]),
           lambda c: c.add_constraint("c", shape=(2,), lower=[0.0, 2.0], upper=[1.0, 1.0]),
           lambda c: c.add_data("d__x"),
           lambda c: c.add_objective("f", scale=1.0, bogus=True)]
    for k, f in enumerate(bad):
        with pytest.raises(ValueError):
            f(cg.Component())
    c = cg.Component()
    c.add_input("x", shape=(2,), lower=[1.0, 2.0], upper=[3.0, 4.0], label="state")
    c.add_input("u", value=0.5, lower=0.0, upper=1.0, units="N", scale=2.0)
    c.add_constraint("c", lower=-1.0, upper=np.inf)
    lo, hi = c.input_bounds()
    assert list(lo) == [1.0, 2.0, 0.0] and list(hi) == [3.0, 4.0, 1.0]
    assert c._inputs.meta["x"]["value"] == 0.0     # unset: amigo's default
    assert c._cons.meta["c"]["lower"] == -1.0 and c._cons.meta["c"]["upper"] == np.inf
