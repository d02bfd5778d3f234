"""Expression DAG for component code generation.

A component's `compute()` builds its objective and constraints from leaf
expressions (its inputs, data and constants) with Python operators and the
unary functions of amigo's modelling layer (amigo/unary_operations.py:1-123,
amigo/expressions.py:386-708 for the operator set).  Here every expression
is a node of one DAG with hash-consing: structurally equal sub-expressions
are the same node, so common sub-expressions are shared by construction and
the emitted code evaluates each once.  Constant folding and the identities
x + 0, x * 1, x * 0 keep derivative expressions small.

`gradient(L, xs)` differentiates by reverse accumulation over the DAG and
returns one expression per variable; `hessian(grad, xs)` differentiates each
gradient entry again (forward-over-reverse symbolically), giving the lower
triangle.  Derivatives are ordinary nodes of the same DAG, so the emitter
(`emit.py`) writes one straight-line program for values, gradient and
Hessian with all shared terms computed once.
"""
import math
import numbers


class Node:
    """One DAG node: op in {"const", "var", "data", "add", "mul", "div",
    "neg", "pow", "<unary function>"}; args are child nodes; `key` is the
    hash-consing key."""

    __slots__ = ("op", "args", "val", "key", "id", "__weakref__")

    def __init__(self, op, args, val, key, id_):
        self.op = op
        self.args = args
        self.val = val
        self.key = key
        self.id = id_


class Graph:
    """Node factory with hash-consing and algebraic simplification."""

    def __init__(self):
        self.table = {}
        self.nodes = []

    def _make(self, op, args=(), val=None):
        key = (op, tuple(a.id for a in args), val)
        n = self.table.get(key)
        if n is None:
            n = Node(op, tuple(args), val, key, len(self.nodes))
            self.table[key] = n
            self.nodes.append(n)
        return n

    # leaves
    def const(self, v):
        v = float(v)
        if v == 0.0:
            v = 0.0   # one zero (no -0.0 node)
        return self._make("const", (), v)

    def var(self, i):
        return self._make("var", (), int(i))

    def data(self, i):
        return self._make("data", (), int(i))

    def alpha(self):
        return self._make("alpha", (), None)

    # arithmetic with simplification
    @staticmethod
    def _c(n):
        return n.val if n.op == "const" else None

    def add(self, a, b):
        ca, cb = self._c(a), self._c(b)
        if ca is not None and cb is not None:
            return self.const(ca + cb)
        if ca == 0.0:
            return b
        if cb == 0.0:
            return a
        if a.id > b.id:   # canonical order: a + b == b + a
            a, b = b, a
        return self._make("add", (a, b))

    def neg(self, a):
        ca = self._c(a)
        if ca is not None:
            return self.const(-ca)
        if a.op == "neg":
            return a.args[0]
        return self._make("neg", (a,))

    def sub(self, a, b):
        return self.add(a, self.neg(b))

    def mul(self, a, b):
        ca, cb = self._c(a), self._c(b)
        if ca is not None and cb is not None:
            return self.const(ca * cb)
        if ca == 0.0 or cb == 0.0:
            return self.const(0.0)
        if ca == 1.0:
            return b
        if cb == 1.0:
            return a
        if ca == -1.0:
            return self.neg(b)
        if cb == -1.0:
            return self.neg(a)
        if a.id > b.id:
            a, b = b, a
        return self._make("mul", (a, b))

    def div(self, a, b):
        ca, cb = self._c(a), self._c(b)
        if cb is not None:
            if cb == 1.0:
                return a
            if ca is not None:
                return self.const(ca / cb)
        if ca == 0.0:
            return self.const(0.0)
        return self._make("div", (a, b))

    def pow(self, a, p):
        """a ** p for a real constant p."""
        p = float(p)
        ca = self._c(a)
        if ca is not None:
            return self.const(ca ** p)
        if p == 0.0:
            return self.const(1.0)
        if p == 1.0:
            return a
        if p == 2.0:
            return self.mul(a, a)
        return self._make("pow", (a,), p)

    def func(self, name, a):
        ca = self._c(a)
        if ca is not None and name in _PY_FUNCS:
            return self.const(_PY_FUNCS[name](ca))
        return self._make(name, (a,))

    def bfunc(self, name, a, b):
        """Binary functions: atan2(a, b); min2 / max2 (a if a < b, resp.
        a > b, else b, the derivative following the chosen argument); lt /
        gt (1.0 where a < b, resp. a > b, else 0.0; derivative 0)."""
        ca, cb = self._c(a), self._c(b)
        if ca is not None and cb is not None:
            return self.const(_PY_BFUNCS[name](ca, cb))
        return self._make(name, (a, b))

    def passive(self, a):
        """The value of a with zero derivative (amigo's passive)."""
        if a.op == "const" or a.op == "passive":
            return a
        return self._make("passive", (a,))


_PY_FUNCS = {
    "sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp,
    "log": math.log, "sqrt": math.sqrt, "tanh": math.tanh, "sinh": math.sinh,
    "cosh": math.cosh, "asin": math.asin, "acos": math.acos, "atan": math.atan,
    "log10": math.log10, "fabs": math.fabs, "asinh": math.asinh, "acosh": math.acosh,
    "atanh": math.atanh,
}
UNARY = tuple(_PY_FUNCS)
_PY_BFUNCS = {
    "atan2": math.atan2,
    "min2": lambda a, b: a if a < b else b,
    "max2": lambda a, b: a if a > b else b,
    "lt": lambda a, b: 1.0 if a < b else 0.0,
    "gt": lambda a, b: 1.0 if a > b else 0.0,
}


class Expr:
    """User-facing expression: a Node plus the Graph it lives in, with the
    Python operators of amigo's expression layer."""

    __slots__ = ("g", "n")

    def __init__(self, g, n):
        self.g = g
        self.n = n

    def _lift(self, o):
        if isinstance(o, Expr):
            return o.n
        if isinstance(o, numbers.Real):
            return self.g.const(o)
        raise TypeError("cannot combine an expression with %r" % type(o))

    def __add__(self, o):
        return Expr(self.g, self.g.add(self.n, self._lift(o)))

    __radd__ = __add__

    def __sub__(self, o):
        return Expr(self.g, self.g.sub(self.n, self._lift(o)))

    def __rsub__(self, o):
        return Expr(self.g, self.g.sub(self._lift(o), self.n))

    def __mul__(self, o):
        return Expr(self.g, self.g.mul(self.n, self._lift(o)))

    __rmul__ = __mul__

    def __truediv__(self, o):
        return Expr(self.g, self.g.div(self.n, self._lift(o)))

    def __rtruediv__(self, o):
        return Expr(self.g, self.g.div(self._lift(o), self.n))

    def __neg__(self):
        return Expr(self.g, self.g.neg(self.n))

    def __pos__(self):
        return self

    def __pow__(self, p):
        if isinstance(p, Expr):
            # a ** b = exp(b log a)
            return Expr(self.g, self.g.func("exp", self.g.mul(p.n, self.g.func("log", self.n))))
        if not isinstance(p, numbers.Real):
            raise TypeError("exponent must be a number or an expression")
        return Expr(self.g, self.g.pow(self.n, p))


def _unary(name):
    def f(x):
        if isinstance(x, Expr):
            return Expr(x.g, x.g.func(name, x.n))
        return _PY_FUNCS[name](float(x))
    f.__name__ = name
    f.__doc__ = "%s of an expression (or of a number)." % name
    return f


sin, cos, tan, exp, log, sqrt, tanh = (_unary(k) for k in
                                       ("sin", "cos", "tan", "exp", "log", "sqrt", "tanh"))
sinh, cosh, asin, acos, atan, log10, fabs = (_unary(k) for k in
                                             ("sinh", "cosh", "asin", "acos", "atan",
                                              "log10", "fabs"))
asinh, acosh, atanh = (_unary(k) for k in ("asinh", "acosh", "atanh"))
abs_ = fabs


def _binary(name):
    def f(a, b):
        if not isinstance(a, Expr) and not isinstance(b, Expr):
            return _PY_BFUNCS[name](float(a), float(b))
        e = a if isinstance(a, Expr) else b
        return Expr(e.g, e.g.bfunc(name, e._lift(a), e._lift(b)))
    f.__name__ = name
    f.__doc__ = "%s of two expressions (or numbers)." % name
    return f


atan2, min2, max2 = (_binary(k) for k in ("atan2", "min2", "max2"))


def passive(x):
    """x without derivative (amigo's passive)."""
    if isinstance(x, Expr):
        return Expr(x.g, x.g.passive(x.n))
    return float(x)


# ---------------------------------------------------------------- derivatives
def _partials(g, n):
    """Local partial derivatives d n / d args[k] as nodes."""
    op, a = n.op, n.args
    if op == "add":
        return (g.const(1.0), g.const(1.0))
    if op == "neg":
        return (g.const(-1.0),)
    if op == "mul":
        return (a[1], a[0])
    if op == "div":
        # d(u/v)/du = 1/v, d(u/v)/dv = -(u/v)/v
        inv = g.div(g.const(1.0), a[1])
        return (inv, g.neg(g.div(n, a[1])))
    if op == "pow":
        p = n.val
        return (g.mul(g.const(p), g.pow(a[0], p - 1.0)),)
    x = a[0]
    if op == "sin":
        return (g.func("cos", x),)
    if op == "cos":
        return (g.neg(g.func("sin", x)),)
    if op == "tan":
        c = g.func("cos", x)
        return (g.div(g.const(1.0), g.mul(c, c)),)
    if op == "exp":
        return (n,)
    if op == "log":
        return (g.div(g.const(1.0), x),)
    if op == "log10":
        return (g.div(g.const(1.0 / math.log(10.0)), x),)
    if op == "sqrt":
        return (g.div(g.const(0.5), n),)
    if op == "tanh":
        return (g.sub(g.const(1.0), g.mul(n, n)),)
    if op == "sinh":
        return (g.func("cosh", x),)
    if op == "cosh":
        return (g.func("sinh", x),)
    if op == "asin":
        return (g.div(g.const(1.0), g.func("sqrt", g.sub(g.const(1.0), g.mul(x, x)))),)
    if op == "acos":
        return (g.neg(g.div(g.const(1.0), g.func("sqrt", g.sub(g.const(1.0), g.mul(x, x))))),)
    if op == "atan":
        return (g.div(g.const(1.0), g.add(g.const(1.0), g.mul(x, x))),)
    if op == "asinh":
        return (g.div(g.const(1.0), g.func("sqrt", g.add(g.mul(x, x), g.const(1.0)))),)
    if op == "acosh":
        return (g.div(g.const(1.0), g.func("sqrt", g.sub(g.mul(x, x), g.const(1.0)))),)
    if op == "atanh":
        return (g.div(g.const(1.0), g.sub(g.const(1.0), g.mul(x, x))),)
    if op == "atan2":
        # d atan2(y, x) = (x dy - y dx) / (x^2 + y^2)
        y, xx = a
        r2 = g.add(g.mul(y, y), g.mul(xx, xx))
        return (g.div(xx, r2), g.neg(g.div(y, r2)))
    if op in ("min2", "max2"):
        s = g.bfunc("lt" if op == "min2" else "gt", a[0], a[1])
        return (s, g.sub(g.const(1.0), s))
    if op in ("lt", "gt"):
        return (g.const(0.0), g.const(0.0))
    if op == "passive":
        return (g.const(0.0),)
    if op == "fabs":
        return (g._make("sign", (x,)),)
    if op == "sign":
        return (g.const(0.0),)
    raise ValueError("no derivative rule for %s" % op)


def _topo(roots):
    """Nodes reachable from roots, children before parents."""
    seen, order, stack = set(), [], []
    for r in roots:
        stack.append((r, False))
    while stack:
        n, done = stack.pop()
        if done:
            order.append(n)
            continue
        if n.id in seen:
            continue
        seen.add(n.id)
        stack.append((n, True))
        for c in n.args:
            if c.id not in seen:
                stack.append((c, False))
    return order


def gradient(g, f, xs):
    """d f / d x for every leaf node x in xs (reverse accumulation)."""
    order = _topo([f])
    adj = {f.id: g.const(1.0)}
    for n in reversed(order):
        a = adj.get(n.id)
        if a is None or not n.args:
            continue
        for c, p in zip(n.args, _partials(g, n)):
            t = g.mul(a, p)
            adj[c.id] = g.add(adj[c.id], t) if c.id in adj else t
    zero = g.const(0.0)
    return [adj.get(x.id, zero) for x in xs]


def hessian(g, grad, xs):
    """Lower triangle H[i][j] (j <= i) of the derivatives of grad[i] with
    respect to xs[j]."""
    return [gradient(g, grad[i], xs[: i + 1]) for i in range(len(xs))]
