"""CPU evaluation of amigo's serialized expression trees.

TEST INFRASTRUCTURE ONLY (the checker for components imported from amigo's
own serialized form; imported by tests/ and the fixture script, never by
the package).

amigo's Component.serialize (amigo/component.py:552-574) writes each
objective, constraint entry and the Lagrangian as nested tuples of the node
classes in amigo/expressions.py:
  ("const", name, value, type)            ConstNode, :37-61
  ("var", name, shape, type, active)      VarNode, :64-85
  ("index", expr, index)                  IndexNode, :88-111 (int or (i, j))
  ("passive", expr)                       PassiveNode, :114-132
  ("unary", op, expr)                     UnaryNode, :135-174 ("-" or A2D::op)
  ("binary", op, left, right)             BinaryNode, :177-226
                                          (+ - * /, ** as A2D::pow, atan2,
                                           min2, max2)
The generated C++ evaluates them with A2D's scalar functions, which are the
C math library's (sin, exp, pow, ...); this module evaluates them with
Python's math module in double precision.  A component's Lagrangian is
alpha__ * objective + sum_k lam_<constraint>__[k] * c_k
(amigo/component.py:775-801).
"""
import math

import numpy as np

_UNARY = {
    "-": lambda a: -a, "sin": math.sin, "cos": math.cos, "tan": math.tan,
    "asin": math.asin, "acos": math.acos, "atan": math.atan, "sinh": math.sinh,
    "cosh": math.cosh, "tanh": math.tanh, "asinh": math.asinh, "acosh": math.acosh,
    "atanh": math.atanh, "exp": math.exp, "log": math.log, "log10": math.log10,
    "sqrt": math.sqrt, "fabs": abs,
}


def _binary(op, a, b):
    if op == "+":
        return a + b
    if op == "-":
        return a - b
    if op == "*":
        return a * b
    if op == "/":
        return a / b
    if op == "**":
        return math.pow(a, b)
    if op == "atan2":
        return math.atan2(a, b)
    if op == "min2":
        return min(a, b)
    if op == "max2":
        return max(a, b)
    raise ValueError("unknown binary operation %r" % op)


def evaluate(tree, env, frozen=None):
    """Value of one serialized expression; env maps variable names to
    floats or numpy arrays (inputs, data, multipliers, alpha__) and
    constant names to their values.  Passive subexpressions (values that
    amigo's derivatives treat as constants) are evaluated in `frozen` when
    it is given, so differences taken around a point hold them at that
    point."""
    kind = tree[0]
    if kind == "const":
        name, value = tree[1], tree[2]
        if name is not None and name in env:
            return float(env[name])
        return float(value)
    if kind == "var":
        return env[tree[1]]
    if kind == "index":
        a = evaluate(tree[1], env, frozen)
        idx = tree[2]
        return float(a[tuple(idx)] if isinstance(idx, (list, tuple)) else a[idx])
    if kind == "passive":
        return evaluate(tree[1], env if frozen is None else frozen)
    if kind == "unary":
        return _UNARY[tree[1]](evaluate(tree[2], env, frozen))
    if kind == "binary":
        return _binary(tree[1], evaluate(tree[2], env, frozen),
                       evaluate(tree[3], env, frozen))
    raise ValueError("unknown node %r" % (kind,))


def _shape(s):
    if s is None:
        return ()
    return tuple(int(v) for v in (s if isinstance(s, (list, tuple)) else [s]))


def _size(s):
    return int(np.prod(_shape(s))) if _shape(s) else 1


def _by_key(d, key):
    return d[key] if key in d else d[str(key)]


def environment(data, x, dvals, alpha):
    """Names -> values for a component serialized by amigo: `x` holds the
    inputs in declaration order (flattened) and then one multiplier per
    constraint entry; `dvals` the data in declaration order."""
    env = {"alpha__": float(alpha)}
    for name, c in data["constants"].items():
        env[name] = float(c["meta"]["value"])
    i = 0
    for group, pre in ((data["inputs"], ""), (data["constraints"], "lam_")):
        for name, c in group.items():
            sh = _shape(c["meta"]["shape"])
            n = _size(sh)
            v = np.asarray(x[i:i + n], dtype=np.float64)
            key = pre + name + ("__" if pre else "")
            env[key] = v.reshape(sh) if sh else float(v[0])
            i += n
    j = 0
    for name, c in data["data"].items():
        sh = _shape(c["meta"]["shape"])
        n = _size(sh)
        v = np.asarray(dvals[j:j + n], dtype=np.float64)
        env[name] = v.reshape(sh) if sh else float(v[0])
        j += n
    return env


def lagrangian(data, x, dvals, alpha, key=0, x_frozen=None):
    """The serialized Lagrangian (amigo's own tree) at (x, dvals, alpha);
    with x_frozen, its passive subexpressions are taken at x_frozen."""
    frozen = (None if x_frozen is None else
              environment(data, x_frozen, dvals, alpha))
    return evaluate(_by_key(data["lagrangian"], key), environment(data, x, dvals, alpha),
                    frozen)


def num_vars(data):
    return (sum(_size(c["meta"]["shape"]) for c in data["inputs"].values())
            + sum(_size(c["meta"]["shape"]) for c in data["constraints"].values()))


def num_data(data):
    return sum(_size(c["meta"]["shape"]) for c in data["data"].values())
