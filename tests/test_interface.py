"""Drop-in interface coverage (CPU only; skipped where the reference
sources are absent): every method that the reference's interior-point
driver (amigo/algorithm/**.py) calls on its InteriorPointOptimizer backend
and on its linear solver exists on amigo_b200's InteriorPointOptimizer and
B200Solver, and accepts the number of positional arguments the call sites
pass."""
import ast
import glob
import inspect
import os

import pytest

from amigo_b200.ipm import InteriorPointOptimizer
from amigo_b200.solver import B200Solver

REF = os.environ.get("AMIGO_REF_ROOT", "/root/reference")
ALG = os.path.join(REF, "amigo", "algorithm")
needs_ref = pytest.mark.skipif(not os.path.isdir(ALG), reason="reference sources absent")


def _receiver(node):
    """Dotted name of an attribute chain (self.optimizer, opt.optimizer...)."""
    parts = []
    while isinstance(node, ast.Attribute):
        parts.append(node.attr)
        node = node.value
    if isinstance(node, ast.Name):
        parts.append(node.id)
    return ".".join(reversed(parts))


def _calls(receivers, skip_dirs=()):
    """{method: set of (positional count, keyword names)} over the driver's
    call sites whose receiver is one of `receivers`."""
    out = {}
    for path in glob.glob(os.path.join(ALG, "**", "*.py"), recursive=True):
        if any(os.sep + d + os.sep in path for d in skip_dirs):
            continue
        tree = ast.parse(open(path).read())
        for n in ast.walk(tree):
            if not (isinstance(n, ast.Call) and isinstance(n.func, ast.Attribute)):
                continue
            if _receiver(n.func.value) not in receivers:
                continue
            if any(isinstance(a, ast.Starred) for a in n.args):
                continue
            out.setdefault(n.func.attr, set()).add(
                (len(n.args), tuple(sorted(k.arg for k in n.keywords if k.arg))))
    return out


def _check(cls, calls, skip=()):
    missing, bad = [], []
    for name, forms in sorted(calls.items()):
        if name in skip:
            continue
        fn = getattr(cls, name, None)
        if fn is None:
            missing.append(name)
            continue
        sig = inspect.signature(fn)
        params = list(sig.parameters.values())[1:]
        pos = [p for p in params if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)]
        names = {p.name for p in params}
        var_pos = any(p.kind == p.VAR_POSITIONAL for p in params)
        var_kw = any(p.kind == p.VAR_KEYWORD for p in params)
        for npos, kws in forms:
            need = [p for p in pos[npos:] if p.default is p.empty and p.name not in kws]
            if (npos > len(pos) and not var_pos) or need or \
                    (not var_kw and any(k not in names for k in kws)):
                bad.append((name, npos, kws))
    return missing, bad


@needs_ref
def test_optimizer_backend_methods_present():
    calls = _calls({"self.optimizer", "opt.optimizer", "self.opt.optimizer"})
    assert len(calls) >= 30
    missing, bad = _check(InteriorPointOptimizer, calls)
    assert not missing, missing
    assert not bad, bad


@needs_ref
def test_linear_solver_methods_present():
    # the solver implementations under solvers/ call their own wrapped
    # backends through `self.solver`: the contract is the driver's calls
    calls = _calls({"self.solver", "opt.solver", "solver", "self.opt.solver"},
                   skip_dirs=("solvers",))
    assert {"factor", "solve"} <= set(calls)
    # MUMPS internals are not part of the solver contract; `solver.lower()`
    # is the solver-name string being normalised (problem_setup.py)
    missing, bad = _check(B200Solver, calls, skip={"_mumps", "lower"})
    assert not missing, missing
    assert not bad, bad
