"""Device code generation for component groups (amigo_b200.codegen), CPU
part: the generated evaluators, compiled for the host from the same source
as the device modules, against the numpy restatements of the benchmark
models (oracle/cartpole_oracle.py, oracle/simp2d_oracle.py) and against
central finite differences; the assembled KKT pattern against the
hand-written models'; the JSON wire format round trip."""
import json

import numpy as np
import pytest

from amigo_b200 import codegen as cg
from amigo_b200.problems import components as C
from amigo_b200.problems.cartpole import CartPole
from amigo_b200.problems.simp2d import Simp2D
from oracle import cartpole_oracle as CO
from oracle import simp2d_oracle as SO


def test_cartpole_generated_matches_oracle():
    m = CartPole(N=20, seed=1)
    G = C.cartpole_model(m)
    assert np.array_equal(G.rowp, m.rowp) and np.array_equal(G.cols, m.cols)
    x = m.x0 + 0.1 * np.random.RandomState(0).randn(m.n)
    g, v = G.host_derivatives(x, 0.7)
    gw, vw = CO.gradient(m, x, 0.7), CO.hessian_values(m, x, 0.7)
    assert np.abs(g - gw).max() <= 1e-13 * np.abs(gw).max()
    assert np.abs(v - vw).max() <= 1e-13 * np.abs(vw).max()


def test_simp2d_generated_matches_oracle():
    m = Simp2D(8, 4, seed=1)
    G = C.simp2d_model(m)
    assert np.array_equal(G.rowp, m.rowp) and np.array_equal(G.cols, m.cols)
    r = np.random.RandomState(0)
    x = r.randn(m.n) * 0.3
    x[m.rt0:m.rt0 + m.nnodes] = 0.2 + 0.6 * r.rand(m.nnodes)
    x[m.re0:m.re0 + m.nelems] = 0.2 + 0.6 * r.rand(m.nelems)
    g, v = G.host_derivatives(x, 0.9)
    gw, vw = SO.gradient_fixed(m, x, 0.9), SO.hessian_values(m, x)
    assert np.abs(g - gw).max() <= 1e-13 * np.abs(gw).max()
    assert np.abs(v - vw).max() <= 1e-13 * np.abs(vw).max()
    # the volume multiplier is shared by every element: summed, not coloured
    vol = [gr for gr in G.groups if gr.name == "volume"][0]
    assert vol.kred == 1 and len(vol.color_ptr) == 2


class AllFunctions(cg.Component):
    """Every operator and unary function of the expression layer."""

    def __init__(self):
        super().__init__()
        self.add_constant("c", 1.5)
        self.add_data("w", shape=2)
        self.add_input("a")
        self.add_input("b", shape=2)
        self.add_constraint("r", shape=3)
        self.add_objective("f")

    def compute(self):
        a, b, w = self.inputs["a"], self.inputs["b"], self.data["w"]
        c = self.constants["c"]
        self.objective["f"] = (cg.sin(a) * cg.cos(b[0]) + cg.exp(0.3 * b[1]) +
                               cg.log(2.0 + a * a) + cg.sqrt(1.0 + b[0] ** 2) +
                               cg.tanh(a - b[1]) + a ** 3.0 / (1.0 + b[1] ** 2) +
                               cg.atan(w[0] * a) + c * cg.sinh(0.2 * b[0]))
        self.constraints["r"] = [a * b[0] - w[1], cg.cosh(0.1 * b[1]) - 2.0 / (3.0 + a * a),
                                 cg.tan(0.2 * a) + cg.asin(0.3 * cg.sin(b[0])) +
                                 cg.acos(0.2 * cg.cos(b[1])) + cg.log10(2.0 + b[1] ** 2) +
                                 b[0] ** 0.5 * 0.0 + (1.0 + a * a) ** 1.7]


def test_generated_derivatives_match_finite_differences():
    comp = AllFunctions()
    ev = cg.host_evaluator(comp, "allf")
    r = np.random.RandomState(4)
    q = np.concatenate([[0.4], [0.7, -0.3], r.randn(3)])
    d = np.array([0.8, 0.25])
    alpha = 1.3
    g, H, obj = ev(q, d, alpha)
    # the Lagrangian from the host evaluator's objective and gradient wrt
    # the multipliers (= the constraint values): L = alpha f + lam . c
    def lag(qq):
        gg, _, f = ev(qq, d, alpha)
        return alpha * f + qq[3:] @ gg[3:]
    eps = 1e-6
    for i in range(len(q)):
        e = np.zeros(len(q))
        e[i] = eps
        fd = (lag(q + e) - lag(q - e)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-7 * max(1.0, abs(g[i])), (i, fd, g[i])
        gp, _, _ = ev(q + e, d, alpha)
        gm, _, _ = ev(q - e, d, alpha)
        col = (gp - gm) / (2 * eps)
        assert np.abs(col - H[:, i]).max() <= 1e-6 * max(1.0, np.abs(H).max()), i
    assert np.allclose(H, H.T, rtol=0, atol=1e-12)


def test_wire_format_round_trip():
    """serialize -> JSON -> deserialize rebuilds a component whose generated
    derivatives agree to rounding (the rebuilt DAG may accumulate adjoints
    in another order), without the defining Python class."""
    for comp, q, d in ((C.TrapezoidInterval(), np.linspace(-0.5, 0.9, 14), [0.02, 0.3]),
                       (AllFunctions(), np.array([0.4, 0.7, -0.3, 0.2, -0.1, 0.5]), [0.8, 0.25])):
        s = json.dumps(comp.serialize())
        back = cg.Component.deserialize(json.loads(s))
        e1 = cg.host_evaluator(comp, "orig")
        e2 = cg.host_evaluator(back, "back")
        a, b = e1(q, np.array(d), 0.9), e2(q, np.array(d), 0.9)
        for u, w in zip(a[:2], b[:2]):
            assert np.abs(u - w).max() <= 1e-14 * max(1.0, np.abs(u).max())
        assert abs(a[2] - b[2]) <= 1e-14 * max(1.0, abs(a[2]))


def test_declaration_errors():
    class Bad(cg.Component):
        def __init__(self):
            super().__init__()
            self.add_input("x")
            self.add_constraint("c", shape=2)

        def compute(self):
            self.constraints["c"] = [self.inputs["x"]]   # one entry for two

    with pytest.raises(ValueError):
        Bad().build()
    with pytest.raises(ValueError):
        cg.Group(C.BoundaryState(), np.zeros((3, 5), np.int32))


def test_model_wire_format_round_trip():
    """A whole problem as a request carries it: GeneratedModel.serialize ->
    JSON -> deserialize gives the same KKT pattern, multiplier indicator,
    bounds, fixed rows and start point, and derivatives equal to rounding;
    vectors round-trip through serialize_vectors."""
    m = CartPole(N=12, seed=3)
    G = C.cartpole_model(m)
    s = json.dumps(G.serialize())
    B = cg.GeneratedModel.deserialize(json.loads(s))
    assert B.n == G.n and np.array_equal(B.rowp, G.rowp) and np.array_equal(B.cols, G.cols)
    assert np.array_equal(B.mult, G.mult) and np.array_equal(B.fixed, G.fixed)
    assert np.array_equal(B.lower, G.lower) and np.array_equal(B.upper, G.upper)
    x = m.x0 + 0.05 * np.random.RandomState(2).randn(m.n)
    g1, v1 = G.host_derivatives(x, 0.8)
    g2, v2 = B.host_derivatives(x, 0.8)
    assert np.abs(g1 - g2).max() <= 1e-14 * np.abs(g1).max()
    assert np.abs(v1 - v2).max() <= 1e-14 * np.abs(v1).max()
    vec = cg.GeneratedModel.serialize_vectors({"x": ("state", x), "p": ("data", np.arange(3.0))})
    back = cg.GeneratedModel.deserialize_vectors(json.loads(json.dumps(vec)))
    assert back["x"][0] == "state" and np.array_equal(back["x"][1], x)
    with pytest.raises(ValueError):
        cg.GeneratedModel.serialize_vectors({"y": ("bogus", x)})
