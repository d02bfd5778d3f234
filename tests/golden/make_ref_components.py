"""Generate tests/golden/ref_components.json: components defined by the
reference's own examples, serialized by the reference's own front end
(amigo/component.py Component.serialize), with sample points and the value
of each serialized Lagrangian there (oracle/expr_oracle.py).

The example scripts build and solve whole models at import, so only their
component classes are run: the class definitions and the module-level
constant assignments they use are taken from each script's syntax tree and
executed with `am` bound to the reference package (its compiled module
replaced by oracle/ref_optimizer.py's stand-in, which component code does
not touch).  Components that cannot be instantiated without arguments,
define no constraint or objective, or use a node the importer rejects are
listed under "skipped" with the reason.  One more component, defined in this
script with the reference's API, covers the functions the examples do not
use (atan2, min2, max2, asinh, acosh, atanh, passive).

    python tests/golden/make_ref_components.py      # needs the reference sources
"""
import ast
import importlib
import json
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from amigo_b200.codegen import from_amigo  # noqa: E402
from oracle import expr_oracle as X  # noqa: E402
from oracle import ref_optimizer as RO  # noqa: E402

SCRIPTS = ["examples/trajectory/cart/cart_pole.py", "examples/sellar/sellar.py",
           "examples/rosenbrock/rosenbrock.py"]
TEST_PROBLEMS = "examples/test_problems"
MAX_JSON = 200_000      # bytes of one serialized component kept in the fixture


def reference_namespace():
    RO.install()
    comp = importlib.import_module("amigo.component")
    un = importlib.import_module("amigo.unary_operations")
    am = types.SimpleNamespace(Component=comp.Component)
    for k in dir(un):
        if not k.startswith("_"):
            setattr(am, k, getattr(un, k))
    return am


def component_classes(path, am):
    """Component classes of one example script (see module docstring)."""
    tree = ast.parse(open(path).read())
    ns = {"am": am, "np": np, "math": math, "__name__": "reference_example"}
    keep = []
    for node in tree.body:
        if isinstance(node, ast.ClassDef):
            keep.append(node)
        elif (isinstance(node, ast.Assign) and all(isinstance(t, ast.Name) for t in node.targets)
              and not any(isinstance(n, ast.Call) and "Model" in ast.unparse(n.func)
                          for n in ast.walk(node))):
            keep.append(node)
    for node in keep:
        try:
            exec(compile(ast.Module(body=[node], type_ignores=[]), path, "exec"), ns)
        except Exception:
            pass
    return [v for v in ns.values()
            if isinstance(v, type) and issubclass(v, am.Component) and v is not am.Component]


def functions_component(am):
    """A component of this script (not from the examples) that uses every
    function of the reference's expression layer the examples leave out."""

    class AllFunctions(am.Component):
        def __init__(self):
            super().__init__()
            self.add_constant("k", value=0.3)
            self.add_input("a")
            self.add_input("b", shape=(2,))
            self.add_data("w")
            self.add_objective("f")
            self.add_constraint("c", shape=(3,))

        def compute(self):
            a, b, w, k = self.inputs["a"], self.inputs["b"], self.data["w"], self.constants["k"]
            self.objective["f"] = (am.atan2(a, b[0]) + am.min2(a * a, b[1]) + am.max2(a, w * b[0])
                                   + am.asinh(a * w) + am.passive(a) * b[1] * a)
            self.constraints["c"] = [am.acosh(1.5 + b[0] * b[0]), am.atanh(k * a),
                                     am.passive(a) * b[0] + am.fabs(a - b[1])]

    return AllFunctions


def main():
    ref_root = RO.REF_ROOT
    am = reference_namespace()
    scripts = list(SCRIPTS)
    tp = os.path.join(ref_root, TEST_PROBLEMS)
    for d in sorted(os.listdir(tp)):
        f = os.path.join(TEST_PROBLEMS, d, d + ".py")
        if os.path.exists(os.path.join(ref_root, f)):
            scripts.append(f)
    r = np.random.RandomState(0)
    out, skipped = [], {}
    for rel in scripts + ["make_ref_components.py"]:
        classes = ([functions_component(am)] if rel == "make_ref_components.py" else
                   component_classes(os.path.join(ref_root, rel), am))
        for cls in classes:
            key = "%s:%s" % (rel, cls.__name__)
            try:
                data = cls().serialize()
            except Exception as e:
                skipped[key] = "not instantiable without arguments: %s" % type(e).__name__
                continue
            data = json.loads(json.dumps(data))
            if not data["constraints"] and not data["objective"]:
                skipped[key] = "no constraint or objective"
                continue
            text = json.dumps(data)
            if len(text) > MAX_JSON:
                skipped[key] = "serialized form larger than %d bytes" % MAX_JSON
                continue
            try:
                comp = from_amigo(data)
                comp.build()
            except ValueError as e:
                skipped[key] = str(e)
                continue
            nq, nd = X.num_vars(data), X.num_data(data)
            points = []
            for _ in range(2):
                # inside the domains of log/sqrt/asin...: small positive values
                x = 0.2 + 0.6 * r.rand(nq)
                d = 0.5 + r.rand(nd)
                alpha = float(0.5 + r.rand())
                try:
                    L = X.lagrangian(data, x, d, alpha)
                except (ValueError, ZeroDivisionError, OverflowError) as e:
                    skipped[key] = "Lagrangian not finite at the sample: %s" % e
                    break
                points.append(dict(x=x.tolist(), d=d.tolist(), alpha=alpha, lagrangian=L))
            if len(points) == 2:
                out.append(dict(source=rel, cls=cls.__name__, data=data, points=points))
    path = os.path.join(HERE, "ref_components.json")
    with open(path, "w") as f:
        json.dump(dict(components=out, skipped=skipped), f, separators=(",", ":"))
    print("%d components, %d skipped -> %s (%d bytes)"
          % (len(out), len(skipped), path, os.path.getsize(path)))
    for k, v in skipped.items():
        print("  skipped", k, "--", v)


if __name__ == "__main__":
    main()
