"""Component: amigo's per-instance modelling unit, for device code generation.

The declaration API is amigo's (amigo/component.py:639-706): `add_constant`,
`add_input`, `add_data`, `add_constraint`, `add_objective`, and a
`compute()` that assigns `self.constraints[name]` and `self.objective[name]`
from `self.inputs`, `self.data` and `self.constants`.  A component's
variable vector is its inputs (in declaration order, flattened) followed by
one multiplier per constraint entry, the layout amigo's generated code uses
(component.py:1010-1061); its Lagrangian is
    L = alpha * sum(objectives) + sum_k lambda_k c_k
(component.py:775-801).  `build()` runs `compute()` on symbolic leaves and
differentiates L (expr.gradient / expr.hessian); `emit.py` writes the
device code.

A component can also be written to and read from a JSON-compatible dict
(`serialize` / `Component.deserialize`): the expression DAG, shapes and
bounds, so a request can carry its model without the Python class that
defined it (the role of amigo's Model.serialize, amigo/model.py:1624-1740).
"""
import numpy as np

from . import expr as E


def _shape(shape):
    if shape is None:
        return ()
    if isinstance(shape, int):
        return (shape,)
    shape = tuple(int(s) for s in shape)
    if len(shape) > 2:
        raise ValueError("shapes have at most two dimensions")
    return shape


def _size(shape):
    return int(np.prod(shape)) if shape else 1


_META_OPTIONS = ("type", "units", "scale", "label")


def _check_meta(kind, name, shape, kw, value=None, lower=None, upper=None):
    """amigo's declaration checks (amigo/meta.py:24-133): names with a
    double underscore are reserved, unknown options are refused, value and
    bounds are scalars or of the declared shape, lower <= upper, and an
    input's value lies within its bounds."""
    if "__" in name:
        raise ValueError("Name %s cannot contain a double underscore" % name)
    unknown = sorted(set(kw) - set(_META_OPTIONS))
    if unknown:
        raise ValueError("Unknown options: %s" % unknown)
    n = _size(_shape(shape))

    def flat(v, what):
        if v is None:
            return None
        a = np.asarray(v, dtype=np.float64)
        if a.ndim == 0:
            return np.full(n, float(a))
        if a.size != n:
            raise ValueError("%s must be scalar or have shape %s" % (what, _shape(shape)))
        return a.ravel()
    val, lo, hi = flat(value, "value"), flat(lower, "lower"), flat(upper, "upper")
    if lo is not None and hi is not None and np.any(lo > hi):
        raise ValueError("lower bound cannot be greater than upper bound")
    if (kind == "input" and val is not None and lo is not None and hi is not None
            and np.any((val < lo) | (val > hi))):
        raise ValueError("value must be within [lower, upper]")


class _Decl:
    """Ordered declarations of one kind with their shapes and metadata."""

    def __init__(self):
        self.names, self.shapes, self.meta = [], {}, {}

    def add(self, name, shape, **meta):
        if name in self.shapes:
            raise ValueError("%s declared twice" % name)
        self.names.append(name)
        self.shapes[name] = _shape(shape)
        self.meta[name] = meta

    def size(self):
        return sum(_size(self.shapes[k]) for k in self.names)

    def __iter__(self):
        return iter(self.names)

    def __len__(self):
        return len(self.names)


class _Values(dict):
    """name -> expression (scalar) or numpy object array of expressions."""


class _Assign(dict):
    """Targets of compute(): constraints[name] = expr / list / array."""

    def __init__(self, decl):
        super().__init__()
        self.decl = decl

    def __setitem__(self, name, value):
        if name not in self.decl.shapes:
            raise KeyError("%s was not declared" % name)
        super().__setitem__(name, value)


class Component:
    def __init__(self):
        self._const = _Decl()
        self._inputs = _Decl()
        self._data = _Decl()
        self._cons = _Decl()
        self._obj = _Decl()
        self._outs = _Decl()
        self._built = None

    # -- declarations (amigo/component.py:639-706) --------------------------
    # Unset value / bounds are None (amigo's defaults apply: value 0.0,
    # inputs unbounded, constraints equalities at 0); the declarations are
    # checked as amigo's Meta checks them (_check_meta).
    def add_constant(self, name, value, **kw):
        _check_meta("constant", name, None, kw)
        self._const.add(name, None, value=float(value), **kw)

    def add_input(self, name, shape=None, value=None, lower=None, upper=None, **kw):
        _check_meta("input", name, shape, kw, value, lower, upper)
        self._inputs.add(name, shape, value=0.0 if value is None else value,
                         lower=-np.inf if lower is None else lower,
                         upper=np.inf if upper is None else upper, **kw)

    def add_data(self, name, shape=None, value=None, **kw):
        _check_meta("data", name, shape, kw, value)
        self._data.add(name, shape, value=0.0 if value is None else value, **kw)

    def add_constraint(self, name, shape=None, lower=None, upper=None, **kw):
        _check_meta("constraint", name, shape, kw, None, lower, upper)
        self._cons.add(name, shape, lower=0.0 if lower is None else lower,
                       upper=0.0 if upper is None else upper, **kw)

    def add_objective(self, name, **kw):
        _check_meta("objective", name, None, kw)
        self._obj.add(name, None, **kw)

    def add_output(self, name, shape=None, **kw):
        """A model output computed from the inputs and data (amigo's
        add_output); outputs do not enter the Lagrangian."""
        _check_meta("output", name, shape, kw)
        self._outs.add(name, shape, **kw)

    def compute(self):
        raise NotImplementedError

    # -- layout ---------------------------------------------------------------
    @property
    def num_inputs(self):
        return self._inputs.size()

    @property
    def num_constraints(self):
        return self._cons.size()

    @property
    def num_vars(self):
        """Inputs followed by one multiplier per constraint entry."""
        return self.num_inputs + self.num_constraints

    @property
    def num_data(self):
        return self._data.size()

    @property
    def num_outputs(self):
        return self._outs.size()

    def var_names(self):
        """Flattened names of the variable vector, e.g. q[1], lam_res[2]."""
        out = []
        for decl, pre in ((self._inputs, ""), (self._cons, "lam:")):
            for k in decl:
                sh = decl.shapes[k]
                if not sh:
                    out.append(pre + k)
                else:
                    out += [pre + k + str(list(ix)) for ix in np.ndindex(*sh)]
        return out

    def input_bounds(self):
        lo, hi = [], []
        for k in self._inputs:
            m, n = self._inputs.meta[k], _size(self._inputs.shapes[k])
            lo += list(np.broadcast_to(np.asarray(m["lower"], float), (n,)))
            hi += list(np.broadcast_to(np.asarray(m["upper"], float), (n,)))
        return np.array(lo), np.array(hi)

    # -- symbolic build -------------------------------------------------------
    def _leaves(self, g, decl, make, base=0):
        vals, i = _Values(), base
        for k in decl:
            sh = decl.shapes[k]
            n = _size(sh)
            leaves = [E.Expr(g, make(i + t)) for t in range(n)]
            if sh:
                a = np.empty(n, dtype=object)
                a[:] = leaves
                vals[k] = a.reshape(sh)
            else:
                vals[k] = leaves[0]
            i += n
        return vals

    def build(self):
        """Run compute() on symbolic leaves; returns (graph, vars, L, obj)."""
        if self._built is not None:
            return self._built
        g = E.Graph()
        self._g = g
        self.inputs = self._leaves(g, self._inputs, g.var)
        self.data = self._leaves(g, self._data, g.data)
        self.constants = {k: self._const.meta[k]["value"] for k in self._const}
        self.constraints = _Assign(self._cons)
        self.objective = _Assign(self._obj)
        self.outputs = _Assign(self._outs)
        self.compute()
        missing = [k for k in self._cons if k not in self.constraints]
        missing += [k for k in self._outs if k not in self.outputs]
        if missing:
            raise ValueError("compute() left constraints or outputs unset: %s" % missing)
        outs = []
        for k in self._outs:
            sh = self._outs.shapes[k]
            vals = self.outputs[k]
            flat = [vals] if not sh else list(np.asarray(vals, dtype=object).ravel())
            if len(flat) != _size(sh):
                raise ValueError("output %s has %d entries, declared %d"
                                 % (k, len(flat), _size(sh)))
            outs += [self._node(g, v) for v in flat]
        self._out_nodes = outs
        ni = self.num_inputs
        lam = [g.var(ni + t) for t in range(self.num_constraints)]
        xs = [g.var(i) for i in range(ni)] + lam
        lag = g.const(0.0)
        obj = g.const(0.0)
        for k in self._obj:
            obj = g.add(obj, self._node(g, self.objective[k]))
        lag = g.mul(g.alpha(), obj)
        t = 0
        for k in self._cons:
            sh = self._cons.shapes[k]
            vals = self.constraints[k]
            flat = [vals] if not sh else list(np.asarray(vals, dtype=object).ravel())
            if len(flat) != _size(sh):
                raise ValueError("constraint %s has %d entries, declared %d"
                                 % (k, len(flat), _size(sh)))
            for v in flat:
                lag = g.add(lag, g.mul(lam[t], self._node(g, v)))
                t += 1
        self._built = (g, xs, lag, obj)
        return self._built

    @staticmethod
    def _node(g, v):
        if isinstance(v, E.Expr):
            return v.n
        return g.const(float(v))

    # -- wire format ----------------------------------------------------------
    def serialize(self):
        """JSON-compatible dict: declarations and the expression DAG of the
        objective and of every constraint entry."""
        g, xs, lag, obj = self.build()
        roots = [obj]
        cons = []
        for k in self._cons:
            sh = self._cons.shapes[k]
            vals = self.constraints[k]
            flat = [vals] if not sh else list(np.asarray(vals, dtype=object).ravel())
            cons.append([self._node(g, v) for v in flat])
            roots += cons[-1]
        outs = list(self._out_nodes)
        roots += outs
        order = E._topo(roots)
        ids = {n.id: i for i, n in enumerate(order)}
        nodes = [[n.op, [ids[a.id] for a in n.args], n.val] for n in order]
        decl = lambda d: [[k, list(d.shapes[k]), _jsonable(d.meta[k])] for k in d]
        return {"format": "amigo_b200.component/1", "name": type(self).__name__,
                "inputs": decl(self._inputs), "data": decl(self._data),
                "constraints": decl(self._cons), "objective": decl(self._obj),
                "outputs": decl(self._outs),
                "nodes": nodes, "objective_root": ids[obj.id],
                "constraint_roots": [[ids[n.id] for n in c] for c in cons],
                "output_roots": [ids[n.id] for n in outs]}

    @classmethod
    def deserialize(cls, d):
        if d.get("format") != "amigo_b200.component/1":
            raise ValueError("not a serialized component")
        return _Deserialized(d)


def _jsonable(meta):
    out = {}
    for k, v in meta.items():
        if isinstance(v, np.ndarray):
            v = v.tolist()
        if isinstance(v, float) and not np.isfinite(v):
            v = "inf" if v > 0 else "-inf"
        out[k] = v
    return out


def _num(v):
    if v == "inf":
        return np.inf
    if v == "-inf":
        return -np.inf
    return v


class _Deserialized(Component):
    """A component rebuilt from its serialized DAG."""

    def __init__(self, d):
        super().__init__()
        self._d = d
        self._serial_name = d.get("name", "Component")
        for k, sh, meta in d["inputs"]:
            meta = {a: _num(b) for a, b in meta.items()}
            self.add_input(k, sh or None, **meta)
        for k, sh, meta in d["data"]:
            self.add_data(k, sh or None, **meta)
        for k, sh, meta in d["constraints"]:
            meta = {a: _num(b) for a, b in meta.items()}
            self.add_constraint(k, sh or None, **meta)
        for k, sh, meta in d["objective"]:
            self.add_objective(k, **meta)
        for k, sh, meta in d.get("outputs", []):
            self.add_output(k, sh or None, **meta)

    def compute(self):
        g = self._g
        made = []
        for op, args, val in self._d["nodes"]:
            a = [made[i] for i in args]
            if op == "const":
                n = g.const(val)
            elif op == "var":
                n = g.var(val)
            elif op == "data":
                n = g.data(val)
            elif op == "alpha":
                n = g.alpha()
            elif op == "add":
                n = g.add(*a)
            elif op == "mul":
                n = g.mul(*a)
            elif op == "div":
                n = g.div(*a)
            elif op == "neg":
                n = g.neg(*a)
            elif op == "pow":
                n = g.pow(a[0], val)
            elif op in ("atan2", "min2", "max2", "lt", "gt"):
                n = g.bfunc(op, a[0], a[1])
            elif op == "passive":
                n = g.passive(a[0])
            else:
                n = g.func(op, a[0])
            made.append(n)
        ex = lambda i: E.Expr(g, made[i])
        for t, k in enumerate(self._obj):
            # the objectives' sum was serialized; it goes to the first one
            self.objective[k] = ex(self._d["objective_root"]) if t == 0 else 0.0
        for (k, sh, _), roots in zip(self._d["constraints"], self._d["constraint_roots"]):
            vals = [ex(i) for i in roots]
            self.constraints[k] = vals[0] if not sh else vals
        roots = list(self._d.get("output_roots", []))
        for k, sh, _ in self._d.get("outputs", []):
            m = _size(tuple(sh))
            vals = [ex(i) for i in roots[:m]]
            roots = roots[m:]
            self.outputs[k] = vals[0] if not sh else vals
