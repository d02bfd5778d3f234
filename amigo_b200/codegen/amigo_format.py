"""Components serialized by amigo itself, rebuilt for device code generation.

amigo's `Component.serialize()` (amigo/component.py:552-574) writes a
component's declarations (constants, inputs, data, constraints, objective,
outputs with their metadata) and the expression trees that its compute()
built, as nested tuples of the node kinds of amigo/expressions.py:37-227.
`from_amigo(data)` turns that dict (or its JSON) into a `Component` of this
package, so a model that amigo's own front end serialized -- a request on
the wire (amigo/model.py:1624-1740) -- is evaluated by the generated CUDA
gradient and Hessian kernels without the Python class that defined it.

The variable vector keeps amigo's layout: the inputs in declaration order,
then one multiplier per constraint entry; bounds and starting values come
from the metadata with amigo's defaults (inputs unbounded from 0.0,
constraints equalities at 0, amigo/meta.py:7-17 and
amigo/model.py:1362-1366).  Every node kind and function of amigo's
expression layer is taken (amigo/unary_operations.py): constants (named
ones take the component's constant value), variables, indexing, unary
minus, sin cos tan asin acos atan sinh cosh tanh asinh acosh atanh exp log
log10 sqrt fabs, the binary + - * / ** operators, atan2, min2 / max2 (the
derivative follows the chosen argument; on a tie, the second) and passive
subexpressions (value without derivative).  More than one compute()
argument set, a continuation component or an unknown node is rejected with
a ValueError naming it.
"""
import json
import math
import numbers

import numpy as np

from . import expr as E
from .component import Component

_UNARY = {"sin": E.sin, "cos": E.cos, "tan": E.tan, "asin": E.asin, "acos": E.acos,
          "atan": E.atan, "sinh": E.sinh, "cosh": E.cosh, "tanh": E.tanh, "exp": E.exp,
          "log": E.log, "log10": E.log10, "sqrt": E.sqrt, "fabs": E.fabs,
          "asinh": E.asinh, "acosh": E.acosh, "atanh": E.atanh}
_BINARY = {"atan2": E.atan2, "min2": E.min2, "max2": E.max2}


def _shape(s):
    if s is None:
        return None
    t = tuple(int(v) for v in (s if isinstance(s, (list, tuple)) else [s]))
    return t or None


def _bound(v):
    """A metadata value as a float or an array (None: unset)."""
    if v is None:
        return None
    a = np.asarray(v, dtype=np.float64)
    return float(a) if a.ndim == 0 else a


def _by_key(d, key):
    if key in d:
        return d[key]
    if str(key) in d:
        return d[str(key)]
    raise ValueError("no expression for compute() argument set %r" % (key,))


class AmigoComponent(Component):
    """A component rebuilt from amigo's serialized form (see module
    docstring); `name` is amigo's component name."""

    def __init__(self, data):
        super().__init__()
        if isinstance(data, str):
            data = json.loads(data)
        if len(data.get("args", [{}])) != 1:
            raise ValueError("components with several compute() argument sets "
                             "are not supported")
        if data.get("continuation_component"):
            raise ValueError("continuation components are not supported")
        self._src = data
        self.name = data.get("name", "Component")
        for k, c in data["constants"].items():
            self.add_constant(k, c["meta"]["value"])
        for k, c in data["inputs"].items():
            m = c["meta"]
            self.add_input(k, _shape(m.get("shape")), value=_bound(m.get("value")),
                           lower=_bound(m.get("lower")), upper=_bound(m.get("upper")))
        for k, c in data["data"].items():
            m = c["meta"]
            self.add_data(k, _shape(m.get("shape")), value=_bound(m.get("value")))
        for k, c in data["constraints"].items():
            m = c["meta"]
            self.add_constraint(k, _shape(m.get("shape")), lower=_bound(m.get("lower")),
                                upper=_bound(m.get("upper")))
        for k in data["objective"]:
            self.add_objective(k)
        for k, c in data.get("outputs", {}).items():
            self.add_output(k, _shape(c["meta"].get("shape")))

    # -- expression trees ------------------------------------------------------
    def _ev(self, t):
        kind = t[0]
        if kind == "const":
            name, value = t[1], t[2]
            if name is not None and name in self.constants:
                return float(self.constants[name])
            return float(value)
        if kind == "var":
            name = t[1]
            if name in self.inputs:
                return self.inputs[name]
            if name in self.data:
                return self.data[name]
            raise ValueError("unknown variable %r" % (name,))
        if kind == "index":
            a = self._ev(t[1])
            idx = t[2]
            return a[tuple(idx)] if isinstance(idx, (list, tuple)) else a[idx]
        if kind == "unary":
            op = t[1]
            a = self._ev(t[2])
            if op == "-":
                return -a
            if op not in _UNARY:
                raise ValueError("unsupported operation %r" % (op,))
            return _UNARY[op](a)
        if kind == "binary":
            op = t[1]
            a, b = self._ev(t[2]), self._ev(t[3])
            if op == "+":
                return a + b
            if op == "-":
                return a - b
            if op == "*":
                return a * b
            if op == "/":
                return a / b
            if op == "**":
                if isinstance(a, numbers.Real) and isinstance(b, numbers.Real):
                    return math.pow(a, b)
                if isinstance(a, numbers.Real):
                    if a <= 0.0:
                        raise ValueError("a constant base of ** must be positive")
                    return E.exp(b * math.log(a))
                return a ** b
            if op in _BINARY:
                return _BINARY[op](a, b)
            raise ValueError("unsupported operation %r" % (op,))
        if kind == "passive":
            return E.passive(self._ev(t[1]))
        raise ValueError("unsupported node %r" % (kind,))

    def _entries(self, c, key=0):
        """Expression(s) of one constraint / output entry set."""
        e = _by_key(c["expr"]["expr"], key)
        sh = _shape(c["meta"].get("shape"))
        if isinstance(e, list):
            vals = [self._ev(x["expr"]) for x in e]
            a = np.empty(len(vals), dtype=object)
            a[:] = vals
            return a.reshape(sh) if sh else a[0]
        return self._ev(e["expr"])

    def compute(self):
        for k, c in self._src["objective"].items():
            self.objective[k] = self._ev(_by_key(c["expr"]["expr"], 0)["expr"])
        for k, c in self._src["constraints"].items():
            self.constraints[k] = self._entries(c)
        for k, c in self._src.get("outputs", {}).items():
            self.outputs[k] = self._entries(c)


def from_amigo(data):
    """Component of this package from amigo's Component.serialize() output
    (a dict, or its JSON text)."""
    return AmigoComponent(data)
