"""Emit device code for a component's Lagrangian derivatives.

For a component with NQ variables (inputs, then constraint multipliers) and
ND data entries, the emitted struct is

    struct <Sym> {
      static constexpr int NQ, ND;
      template <class Out> __host__ __device__ static void eval(
          const double* q, const double* d, double alpha, Out& out);
      __host__ __device__ static double objective(const double* q,
                                                  const double* d);
    };

`eval` is one straight-line program over the expression DAG: every node the
outputs need is computed once, in topological order, into a local; it calls
out.grad(i, dL/dq_i) for every variable and, when Out::kHess, out.hess(i,
j, d2L/dq_i dq_j) for the non-zero entries of the lower triangle (j <= i).
The Hessian-only nodes sit inside `if constexpr (Out::kHess)`, so the
gradient kernel does not evaluate them.  This is the role of the
`lagrange / gradient / hessian` functions amigo generates per component
(amigo/component.py:1022-1108), written for direct evaluation on the GPU
instead of an automatic-differentiation library's stacks.
"""
import hashlib

from . import expr as E

_FUNCS = {"sin": "sin", "cos": "cos", "tan": "tan", "exp": "exp", "log": "log",
          "sqrt": "sqrt", "tanh": "tanh", "sinh": "sinh", "cosh": "cosh",
          "asin": "asin", "acos": "acos", "atan": "atan", "log10": "log10",
          "fabs": "fabs", "asinh": "asinh", "acosh": "acosh", "atanh": "atanh"}


def _lit(v):
    s = repr(float(v))
    if "e" not in s and "." not in s and "n" not in s:
        s += ".0"
    return s


def _closure(roots, have):
    """Nodes needed by roots, not in `have`, in topological order."""
    out = []
    for n in E._topo(roots):
        if n.id in have or n.op in ("const", "var", "data", "alpha"):
            continue
        out.append(n)
        have.add(n.id)
    return out


def _ref(n):
    if n.op == "const":
        return _lit(n.val)
    if n.op == "var":
        return "q[%d]" % n.val
    if n.op == "data":
        return "d[%d]" % n.val
    if n.op == "alpha":
        return "alpha"
    return "t%d" % n.id


def _expr(n):
    a = [_ref(c) for c in n.args]
    op = n.op
    if op == "add":
        return "%s + %s" % (a[0], a[1])
    if op == "mul":
        return "%s * %s" % (a[0], a[1])
    if op == "div":
        return "%s / %s" % (a[0], a[1])
    if op == "neg":
        return "-%s" % a[0]
    if op == "pow":
        p = n.val
        if p == int(p) and 2 <= p <= 4:
            return " * ".join([a[0]] * int(p))
        if p == -1.0:
            return "1.0 / %s" % a[0]
        if p == 0.5:
            return "sqrt(%s)" % a[0]
        return "pow(%s, %s)" % (a[0], _lit(p))
    if op == "sign":
        return "(%s > 0.0 ? 1.0 : (%s < 0.0 ? -1.0 : 0.0))" % (a[0], a[0])
    if op == "atan2":
        return "atan2(%s, %s)" % (a[0], a[1])
    if op == "min2":
        return "(%s < %s ? %s : %s)" % (a[0], a[1], a[0], a[1])
    if op == "max2":
        return "(%s > %s ? %s : %s)" % (a[0], a[1], a[0], a[1])
    if op == "lt":
        return "(%s < %s ? 1.0 : 0.0)" % (a[0], a[1])
    if op == "gt":
        return "(%s > %s ? 1.0 : 0.0)" % (a[0], a[1])
    if op == "passive":
        return a[0]
    if op in _FUNCS:
        return "%s(%s)" % (_FUNCS[op], a[0])
    raise ValueError("cannot emit %s" % op)


def _stmts(nodes, indent):
    return "".join("%sconst double t%d = %s;\n" % (indent, n.id, _expr(n)) for n in nodes)


def derivatives(comp):
    """(graph, vars, lagrangian, objective, gradient list, hessian rows)."""
    g, xs, lag, obj = comp.build()
    grad = E.gradient(g, lag, xs)
    hess = E.hessian(g, grad, xs)
    return g, xs, lag, obj, grad, hess


def struct_source(comp, sym):
    """C++ source of the evaluator struct `sym` for component `comp`."""
    g, xs, lag, obj, grad, hess = derivatives(comp)
    nq, nd = comp.num_vars, comp.num_data
    have = set()
    gnodes = _closure(grad, have)
    hroots = [h for row in hess for h in row]
    hnodes = _closure(hroots, have)
    onodes = _closure([obj], set())
    out = []
    out.append("struct %s {\n" % sym)
    out.append("  static constexpr int NQ = %d;\n" % nq)
    out.append("  static constexpr int ND = %d;\n" % nd)
    nzh = sum(1 for row in hess for h in row if not (h.op == "const" and h.val == 0.0))
    out.append("  static constexpr int NNZ_HESS = %d;\n" % nzh)
    out.append("  template <class Out>\n")
    out.append("  __host__ __device__ static void eval(const double* __restrict__ q,\n"
               "      const double* __restrict__ d, double alpha, Out& out) {\n")
    out.append("    (void)q; (void)d; (void)alpha;\n")
    out.append(_stmts(gnodes, "    "))
    for i, gi in enumerate(grad):
        out.append("    out.grad(%d, %s);\n" % (i, _ref(gi)))
    out.append("    if constexpr (Out::kHess) {\n")
    out.append(_stmts(hnodes, "      "))
    for i, row in enumerate(hess):
        for j, h in enumerate(row):
            if h.op == "const" and h.val == 0.0:
                continue
            out.append("      out.hess(%d, %d, %s);\n" % (i, j, _ref(h)))
    out.append("    }\n  }\n")
    out.append("  __host__ __device__ static double objective(const double* __restrict__ q,\n"
               "      const double* __restrict__ d) {\n")
    out.append("    (void)q; (void)d;\n")
    out.append(_stmts(onodes, "    "))
    out.append("    return %s;\n  }\n};\n" % _ref(obj))
    return "".join(out)


def sens_source(comp, sym):
    """C++ source of `<sym>_sens`: the outputs and the derivatives a
    post-optimality analysis needs (amigo/algorithm/post_optimization.py),
    dense per instance: out[NO], dgd[NQ * ND] = d(dL/dq_i)/dd_m,
    doq[NO * NQ] = d out_o / dq_i, dod[NO * ND] = d out_o / dd_m."""
    g, xs, lag, obj, grad, hess = derivatives(comp)
    nq, nd, no = comp.num_vars, comp.num_data, comp.num_outputs
    ds = [g.data(m) for m in range(nd)]
    outs = list(comp._out_nodes)
    dgd = [E.gradient(g, gi, ds) for gi in grad]
    doq = [E.gradient(g, o, xs) for o in outs]
    dod = [E.gradient(g, o, ds) for o in outs]
    roots = list(grad) + outs + [h for r in dgd + doq + dod for h in r]
    nodes = _closure(roots, set())
    out = ["struct %s_sens {\n" % sym,
           "  static constexpr int NO = %d;\n" % no,
           "  __host__ __device__ static void eval(const double* __restrict__ q,\n"
           "      const double* __restrict__ d, double alpha, double* out, double* dgd,\n"
           "      double* doq, double* dod) {\n",
           "    (void)q; (void)d; (void)alpha; (void)out; (void)dgd; (void)doq; (void)dod;\n",
           _stmts(nodes, "    ")]
    for o, n in enumerate(outs):
        out.append("    out[%d] = %s;\n" % (o, _ref(n)))
    for i, row in enumerate(dgd):
        for m, n in enumerate(row):
            out.append("    dgd[%d] = %s;\n" % (i * nd + m, _ref(n)))
    for o, row in enumerate(doq):
        for i, n in enumerate(row):
            out.append("    doq[%d] = %s;\n" % (o * nq + i, _ref(n)))
    for o, row in enumerate(dod):
        for m, n in enumerate(row):
            out.append("    dod[%d] = %s;\n" % (o * nd + m, _ref(n)))
    out.append("  }\n};\n")
    return "".join(out)


def module_source(groups, header="codegen_kernels.cuh"):
    """Full CUDA source of a generated module: one evaluator struct and the
    extern "C" launchers (gradient, Hessian, objective) per component
    group.  groups: list of (symbol, component)."""
    parts = ["// Generated by amigo_b200.codegen: component Lagrangian derivatives.\n",
             "#include \"%s\"\n\n" % header]
    for sym, comp in groups:
        parts.append(struct_source(comp, sym))
        parts.append(sens_source(comp, sym))
        parts.append("AB_GEN_ENTRY_POINTS(%s)\n" % sym)
        parts.append("AB_GEN_SENS(%s)\n\n" % sym)
    return "".join(parts)


def source_hash(src):
    return hashlib.sha1(src.encode()).hexdigest()[:16]
