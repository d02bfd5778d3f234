"""A problem assembled from component groups with generated device code.

`GeneratedModel(n, groups, mult, lower, upper, fixed)` is the device-side
counterpart of amigo's OptimizationProblem for this path
(include/optimization_problem.h:596-818): every group is a Component and an
index layout (E instances x NQ global variable indices: the component's
inputs, then its constraint multipliers) plus an E x ND data array.  It
builds
  * the KKT sparsity pattern: every pair of variables that share an
    instance, plus the diagonal, sorted rows (the pattern
    create_csr_from_element_conn builds, include/ordering_utils.h:375-529);
  * per instance, the CSR positions of its NQ x NQ block;
  * a colouring of each group's instances such that instances of one colour
    share no variable (greedy, in instance order);
and compiles the generated evaluators into a shared library
(amigo_b200/_gen/, keyed by a hash of the source; nvcc for sm_100a).  The
device model's gradient / hessian / objective have the interface of the
hand-written device models (amigo_b200/fem.py), so the IPM drivers and
B200Solver take either.
"""
import ctypes
import os
import subprocess

import numpy as np
import scipy.sparse as sp
import torch

from . import emit
from .component import Component

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
CSRC = os.path.join(PKG, "csrc")
GEN_DIR = os.path.join(PKG, "_gen")


class Group:
    def __init__(self, component, idx, data=None, name=None):
        self.comp = component
        self.idx = np.ascontiguousarray(idx, dtype=np.int32)
        nq, nd = component.num_vars, component.num_data
        if self.idx.ndim != 2 or self.idx.shape[1] != nq:
            raise ValueError("index layout must be E x %d" % nq)
        E = self.idx.shape[0]
        if data is None:
            data = np.zeros((E, nd))
        self.data = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(E, nd))
        self.name = name or type(component).__name__
        self.E = E


class Slack(Component):
    """amigo's slack coupling (include/slack_coupling.h:22-80; the Model
    adds one per inequality constraint row, amigo/model.py:975-1010): an
    input s and the constraint res = -s, so that with the row's own
    constraint c the multiplier row reads c(x) - s = 0 and s carries the
    row's bounds."""

    def __init__(self):
        super().__init__()
        self.add_input("s")
        self.add_constraint("res")

    def compute(self):
        self.constraints["res"] = -self.inputs["s"]


def with_slacks(n, groups, mult, lower, upper, rows, row_lower, row_upper, x0=None,
                fixed=(), f=None):
    """GeneratedModel whose multiplier rows `rows` are inequalities
    row_lower <= c(x) <= row_upper: one slack variable per row appended
    after the n variables (bounds [row_lower, row_upper], start 0), coupled
    into its row by a Slack group, and the row's target set to 0.  The
    model's slack_indices / slack_rows give the pairs for
    InteriorPointOptimizer.set_slack_mapping."""
    rows = np.asarray(rows, np.int64)
    ns = len(rows)
    mult = np.asarray(mult, bool)
    if ns and not np.all(mult[rows]):
        raise ValueError("slack rows must be multiplier rows")
    lo = np.asarray(row_lower, float)
    hi = np.asarray(row_upper, float)
    if np.any(lo > hi):
        raise ValueError("lower bound cannot be greater than upper bound")
    sidx = np.arange(n, n + ns)
    lower = np.concatenate([np.asarray(lower, float), lo])
    upper = np.concatenate([np.asarray(upper, float), hi])
    lower[rows] = 0.0
    x0 = None if x0 is None else np.concatenate([np.asarray(x0, float), np.zeros(ns)])
    groups = list(groups)
    if ns:
        groups.append(Group(Slack(), np.stack([sidx, rows], axis=1), name="Slack"))
    m = GeneratedModel(n + ns, groups, np.concatenate([mult, np.zeros(ns, bool)]),
                       lower, upper, fixed=fixed, x0=x0, f=f)
    m.slack_indices = sidx.astype(np.int32)
    m.slack_rows = rows.astype(np.int32)
    return m


def _symbol(name, k):
    s = "".join(ch if ch.isalnum() else "_" for ch in name)
    return "g%d_%s" % (k, s)


def compile_module(src, host=False):
    """Build the generated source (nvcc, sm_100a; or the host compiler for
    the CPU tests) into amigo_b200/_gen/; returns the library path."""
    os.makedirs(GEN_DIR, exist_ok=True)
    h = emit.source_hash(src + ("host" if host else "dev"))
    lib = os.path.join(GEN_DIR, ("gen_host_%s.so" if host else "gen_%s.so") % h)
    if os.path.exists(lib):
        return lib
    cu = os.path.join(GEN_DIR, "gen_%s.%s" % (h, "cpp" if host else "cu"))
    with open(cu, "w") as f:
        f.write(src)
    tmp = lib + ".tmp"
    if host:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + CSRC, cu, "-o", tmp]
    else:
        nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
        if not os.path.exists(nvcc):
            nvcc = "nvcc"
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
               "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "-I" + CSRC,
               "--expt-relaxed-constexpr", cu, "-o", tmp, "-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("generated module failed to compile:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, lib)
    return lib


def greedy_colors(idx, n):
    """Colour instances so that no two of one colour share a variable."""
    E, nq = idx.shape
    color = np.full(E, -1, np.int32)
    # colours already used at each variable, as bit masks (up to 63, then a list)
    used = [0] * n
    for e in range(E):
        m = 0
        for v in idx[e]:
            m |= used[v]
        c = 0
        while m >> c & 1:
            c += 1
        color[e] = c
        bit = 1 << c
        for v in idx[e]:
            used[v] |= bit
    return color


class GeneratedModel:
    def __init__(self, n, groups, mult, lower, upper, fixed=(), x0=None, f=None):
        self.n = int(n)
        self.groups = list(groups)
        self.mult = np.asarray(mult, bool)
        self.lower = np.asarray(lower, float)
        self.upper = np.asarray(upper, float)
        self.fixed = np.ascontiguousarray(np.sort(np.asarray(fixed, np.int64)), dtype=np.int32)
        if x0 is not None:
            self.x0 = np.asarray(x0, float)
        self.syms = [_symbol(gr.name, k) for k, gr in enumerate(self.groups)]
        self._pattern()

    # -- pattern, positions, colours ------------------------------------------
    def _pattern(self):
        n = self.n
        rows, cols = [np.arange(n)], [np.arange(n)]
        for gr in self.groups:
            k = gr.idx.shape[1]
            rows.append(np.repeat(gr.idx, k, axis=1).ravel())
            cols.append(np.tile(gr.idx, (1, k)).ravel())
        r = np.concatenate(rows).astype(np.int64)
        c = np.concatenate(cols).astype(np.int64)
        P = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(n, n))
        P.sum_duplicates()
        P.sort_indices()
        self.rowp = P.indptr.astype(np.int32)
        self.cols = P.indices.astype(np.int32)
        self.nnz = int(self.rowp[-1])
        keys = np.repeat(np.arange(n, dtype=np.int64), np.diff(self.rowp)) * n + \
            self.cols.astype(np.int64)

        def pos(rr, cc):
            q = rr.astype(np.int64) * n + cc.astype(np.int64)
            p = np.searchsorted(keys, q)
            assert np.all(keys[p] == q)
            return p.astype(np.int32)

        for gr in self.groups:
            k = gr.idx.shape[1]
            gr.pos = pos(np.repeat(gr.idx, k, axis=1), np.tile(gr.idx, (1, k))
                         ).reshape(gr.E, k * k)
            # a local variable that is one global variable for every
            # instance (a global multiplier or slack) is summed per instance
            # instead of colouring on it
            shared = [k_ for k_ in range(k) if gr.E > 1 and np.all(gr.idx[:, k_] == gr.idx[0, k_])]
            if len(shared) > 1:
                raise ValueError("group %s: at most one variable may be shared by "
                                 "all instances" % gr.name)
            gr.kred = shared[0] if shared else -1
            cidx = gr.idx if gr.kred < 0 else np.delete(gr.idx, gr.kred, axis=1)
            col = greedy_colors(cidx, n)
            order = np.argsort(col, kind="stable").astype(np.int32)
            counts = np.bincount(col, minlength=int(col.max()) + 1 if gr.E else 0)
            gr.color_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
            gr.color_elems = order
        self.diag_pos = pos(np.arange(n), np.arange(n))
        isf = np.zeros(n, bool)
        isf[self.fixed] = True
        rr = np.repeat(np.arange(n), np.diff(self.rowp))
        zero = (isf[rr] | isf[self.cols]) & (rr != self.cols)
        self.fixed_zero_pos = np.nonzero(zero)[0].astype(np.int32)
        self.fixed_diag_pos = self.diag_pos[self.fixed].astype(np.int32)

    # -- wire format ------------------------------------------------------------
    # A request carries its problem as JSON: the flattened model -- every
    # group's component (its expression DAG, component.serialize), index
    # layout and data, the multiplier indicator, the bounds and the fixed
    # variables -- which is what amigo's Model.initialize produces from the
    # linked, named components that Model.serialize writes
    # (amigo/model.py:1624-1740).  Vectors travel as serialize_vectors
    # writes them: {name: {"kind": ..., "values": [...]}}.
    FORMAT = "amigo_b200.model/1"

    def serialize(self):
        b = lambda a: [None if not np.isfinite(v) else float(v) for v in a]
        d = {"format": self.FORMAT, "n": self.n,
             "groups": [{"name": gr.name, "component": gr.comp.serialize(),
                         "idx": gr.idx.tolist(), "data": gr.data.tolist()}
                        for gr in self.groups],
             "mult": np.nonzero(self.mult)[0].tolist(),
             "lower": b(self.lower), "upper": b(self.upper),
             "fixed": self.fixed.tolist()}
        if hasattr(self, "x0"):
            d["x0"] = [float(v) for v in self.x0]
        return d

    @classmethod
    def deserialize(cls, d):
        from .component import Component
        if d.get("format") != cls.FORMAT:
            raise ValueError("not a serialized model")
        n = int(d["n"])
        groups = [Group(Component.deserialize(g["component"]), np.asarray(g["idx"], np.int32),
                        np.asarray(g["data"], np.float64), name=g["name"])
                  for g in d["groups"]]
        mult = np.zeros(n, bool)
        mult[np.asarray(d["mult"], np.int64)] = True
        lb = lambda a, inf: np.array([inf if v is None else v for v in a], np.float64)
        return cls(n, groups, mult, lb(d["lower"], -np.inf), lb(d["upper"], np.inf),
                   fixed=d.get("fixed", ()), x0=d.get("x0"))

    @staticmethod
    def serialize_vectors(vecs):
        """{name: (kind, array)} -> JSON-compatible dict; kind is "state"
        (n: variables and multipliers), "data" or "output"."""
        out = {}
        for name, (kind, a) in vecs.items():
            if kind not in ("state", "data", "output"):
                raise ValueError("unrecognized vector kind %s" % kind)
            a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
            out[name] = {"kind": kind, "values": [float(v) for v in a.ravel()]}
        return out

    @staticmethod
    def deserialize_vectors(d):
        out = {}
        for name, v in d.items():
            if v.get("kind") not in ("state", "data", "output"):
                raise ValueError("unrecognized vector kind %s" % v.get("kind"))
            out[name] = (v["kind"], np.asarray(v["values"], np.float64))
        return out

    def host_derivatives(self, x, alpha=1.0):
        """Gradient and KKT values assembled on the host from the host build
        of the generated evaluators (test use: no GPU needed)."""
        g = np.zeros(self.n)
        vals = np.zeros(self.nnz)
        for sym, gr in zip(self.syms, self.groups):
            ev = host_evaluator(gr.comp, sym)
            nq = gr.idx.shape[1]
            for e in range(gr.E):
                ge, He, _ = ev(x[gr.idx[e]], gr.data[e], alpha)
                np.add.at(g, gr.idx[e], ge)
                np.add.at(vals, gr.pos[e], He.ravel())
        g[self.fixed] = 0.0
        vals[self.fixed_zero_pos] = 0.0
        vals[self.fixed_diag_pos] = 1.0
        return g, vals

    def host_lagrangian(self, x, alpha=1.0):
        """alpha f(x) + lambda^T c(x) on the host (test use): the objective
        from the host evaluators, c(x) from the gradient's multiplier rows."""
        f = 0.0
        for sym, gr in zip(self.syms, self.groups):
            ev = host_evaluator(gr.comp, sym)
            for e in range(gr.E):
                f += ev(x[gr.idx[e]], gr.data[e], 1.0)[2]
        g, _ = self.host_derivatives(x, alpha)
        return alpha * f + float(x[self.mult] @ g[self.mult])

    def source(self):
        return emit.module_source(list(zip(self.syms, [g.comp for g in self.groups])))

    def device_model(self, device):
        return GeneratedDevice(self, device)


class GeneratedDevice:
    """Uploaded layouts and the loaded generated module; the same calls as
    the hand-written device models: gradient(x, alpha, g) overwrites g,
    hessian(x, alpha, vals) overwrites the KKT values, objective(x, out)."""

    def __init__(self, model, device):
        self.m = model
        self.device = torch.device(device)
        self.lib = ctypes.CDLL(compile_module(model.source()))
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(self.device)
        self.g = []
        for sym, gr in zip(model.syms, model.groups):
            d = dict(idx=t(gr.idx, np.int32), data=t(gr.data, np.float64),
                     pos=t(gr.pos, np.int32), elems=t(gr.color_elems, np.int32),
                     cptr=gr.color_ptr, E=gr.E, kred=int(gr.kred),
                     gk=int(gr.idx[0, gr.kred]) if gr.kred >= 0 else -1,
                     gkk=int(model.diag_pos[gr.idx[0, gr.kred]]) if gr.kred >= 0 else -1,
                     red=torch.zeros(max(gr.E, 1), dtype=torch.float64, device=self.device),
                     obj=torch.zeros(max(gr.E, 1), dtype=torch.float64, device=self.device))
            for what in ("gradient", "hessian", "objective"):
                fn = getattr(self.lib, "%s_%s" % (sym, what))
                fn.restype = ctypes.c_int
                d[what] = fn
            self.g.append(d)
        self.fixed = t(model.fixed, np.int32)
        self.fzero = t(model.fixed_zero_pos, np.int32)
        self.fdiag = t(model.fixed_diag_pos, np.int32)
        for name in ("abgen_fill_at", "abgen_sum"):
            getattr(self.lib, name).restype = ctypes.c_int

    def _s(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    @staticmethod
    def _chk(rc, what):
        if rc != 0:
            raise RuntimeError("generated %s failed (%d)" % (what, rc))

    def _colors(self, d, fn, *args):
        s = self._s()
        base = d["elems"].data_ptr()
        for c in range(len(d["cptr"]) - 1):
            a, b = int(d["cptr"][c]), int(d["cptr"][c + 1])
            self._chk(fn(b - a, ctypes.c_void_p(base + 4 * a), *args, s), "kernel")

    def _reduce_shared(self, d, target, at):
        """target[at] += sum of the group's per-instance shared-variable
        slots, in a fixed order."""
        self._chk(self.lib.abgen_sum(d["E"], ctypes.c_void_p(d["red"].data_ptr()),
                                     ctypes.c_void_p(target.data_ptr() + 8 * at), 1,
                                     self._s()), "shared-variable sum")

    def gradient(self, x, alpha, grad):
        grad.zero_()
        for d in self.g:
            if d["kred"] >= 0:
                d["red"].zero_()
            self._colors(d, d["gradient"], ctypes.c_void_p(d["idx"].data_ptr()),
                         ctypes.c_void_p(d["data"].data_ptr()),
                         ctypes.c_void_p(x.data_ptr()), ctypes.c_double(alpha),
                         ctypes.c_void_p(grad.data_ptr()), ctypes.c_int(d["kred"]),
                         ctypes.c_void_p(d["red"].data_ptr()))
            if d["kred"] >= 0:
                self._reduce_shared(d, grad, d["gk"])
        if len(self.fixed):
            self._chk(self.lib.abgen_fill_at(len(self.fixed), ctypes.c_void_p(self.fixed.data_ptr()),
                                             ctypes.c_double(0.0), ctypes.c_void_p(grad.data_ptr()),
                                             self._s()), "fixed rows")

    def hessian(self, x, alpha, vals):
        vals.zero_()
        for d in self.g:
            if d["kred"] >= 0:
                d["red"].zero_()
            self._colors(d, d["hessian"], ctypes.c_void_p(d["idx"].data_ptr()),
                         ctypes.c_void_p(d["data"].data_ptr()),
                         ctypes.c_void_p(d["pos"].data_ptr()),
                         ctypes.c_void_p(x.data_ptr()), ctypes.c_double(alpha),
                         ctypes.c_void_p(vals.data_ptr()), ctypes.c_int(d["kred"]),
                         ctypes.c_void_p(d["red"].data_ptr()))
            if d["kred"] >= 0:
                self._reduce_shared(d, vals, d["gkk"])
        if len(self.fzero):
            self._chk(self.lib.abgen_fill_at(len(self.fzero), ctypes.c_void_p(self.fzero.data_ptr()),
                                             ctypes.c_double(0.0), ctypes.c_void_p(vals.data_ptr()),
                                             self._s()), "fixed entries")
        if len(self.fdiag):
            self._chk(self.lib.abgen_fill_at(len(self.fdiag), ctypes.c_void_p(self.fdiag.data_ptr()),
                                             ctypes.c_double(1.0), ctypes.c_void_p(vals.data_ptr()),
                                             self._s()), "fixed diagonal")

    def objective(self, x, out):
        """out[0] = the sum of every instance's objective terms."""
        s = self._s()
        for k, d in enumerate(self.g):
            self._chk(d["objective"](d["E"], ctypes.c_void_p(d["idx"].data_ptr()),
                                     ctypes.c_void_p(d["data"].data_ptr()),
                                     ctypes.c_void_p(x.data_ptr()),
                                     ctypes.c_void_p(d["obj"].data_ptr()), s), "objective")
            self._chk(self.lib.abgen_sum(d["E"], ctypes.c_void_p(d["obj"].data_ptr()),
                                         ctypes.c_void_p(out.data_ptr()), int(k > 0), s),
                      "objective sum")

    def launch_count(self):
        self.lib.abgen_launch_count.restype = ctypes.c_longlong
        return int(self.lib.abgen_launch_count())


def host_evaluator(component, sym="comp"):
    """The generated evaluator compiled for the host: returns a function
    (q, d, alpha) -> (gradient, Hessian (NQ x NQ), objective)."""
    return host_evaluators([(sym, component)])[0]


def host_evaluators(pairs):
    """host_evaluator for several (symbol, component) pairs compiled as one
    host module; returns the evaluators in order."""
    lib = ctypes.CDLL(compile_module(emit.module_source(list(pairs)), host=True))
    return [_host_ev(lib, sym, comp) for sym, comp in pairs]


def _host_ev(lib, sym, component):
    fn = getattr(lib, sym + "_eval_host")
    fn.restype = ctypes.c_int
    nq, nd = component.num_vars, component.num_data
    P = ctypes.POINTER(ctypes.c_double)

    def ev(q, d=None, alpha=1.0):
        q = np.ascontiguousarray(q, dtype=np.float64)
        d = np.ascontiguousarray(np.zeros(max(nd, 1)) if d is None else d, dtype=np.float64)
        g = np.zeros(nq)
        H = np.zeros((nq, nq))
        obj = np.zeros(1)
        fn(q.ctypes.data_as(P), d.ctypes.data_as(P), ctypes.c_double(alpha),
           g.ctypes.data_as(P), H.ctypes.data_as(P), obj.ctypes.data_as(P))
        return g, H, float(obj[0])
    return ev
