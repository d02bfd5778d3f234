"""Device-resident CSRMat / Vector / SparseLDL with amigo's interfaces.

These classes mirror the Python-visible API that amigo's pybind module
exposes for the same objects (amigo/amigo.cpp:323-402 for CSRMat and
Vector, 616-694 for SparseLDL), but their numeric data live in HBM as torch
tensors and every numeric operation runs in libamigo_b200.so.  Host copies
exist only where amigo's API hands out numpy arrays.
"""
import ctypes
import enum

import numpy as np
import torch

from . import _lib


class OrderingType(enum.IntEnum):
    """Same values as amigo.OrderingType (include/ordering_utils.h:21)."""
    NESTED_DISSECTION = 0
    AMD = 1
    MULTI_COLOR = 2
    NATURAL = 3
    # amigo.OrderingType.DEFAULT is AMD when METIS is not available
    # (amigo/amigo.cpp:301-311).
    DEFAULT = 1


class SolverType(enum.IntEnum):
    """Same values as amigo.SolverType (amigo/amigo.cpp:611-614)."""
    LDL = 0
    CHOLESKY = 1


def _device(device=None):
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("amigo_b200 needs a CUDA device")
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device(device)


def _stream_ptr(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Vector:
    """amigo.Vector with a host array and a device mirror (HOST_AND_DEVICE).

    ``get_array()`` returns the host numpy array (a view, as amigo's does);
    ``copy_host_to_device`` / ``copy_device_to_host`` synchronise the two.
    Kernels read and write ``self.dev``.
    """

    def __init__(self, size, device=None, dev=None):
        self.device = _device(device) if dev is None else dev.device
        self.size = int(size)
        self.host = np.zeros(self.size)
        self.dev = (torch.zeros(self.size, dtype=torch.float64, device=self.device)
                    if dev is None else dev)

    def get_size(self):
        return self.size

    def get_array(self):
        return self.host

    def __len__(self):
        return self.size

    def __getitem__(self, k):
        return self.host[k]

    def __setitem__(self, k, v):
        self.host[k] = v

    def copy_host_to_device(self):
        self.dev.copy_(torch.from_numpy(self.host))

    def copy_device_to_host(self):
        self.host[:] = self.dev.cpu().numpy()

    def zero(self):
        self.host[:] = 0.0
        self.dev.zero_()


class CSRMat:
    """Square symmetric CSR matrix (both triangles stored) with device values.

    Mirrors amigo.CSRMat(nrows, ncols, rowp, cols, vals) and its
    ``get_nonzero_structure``, ``get_data``, ``copy_data_device_to_host``
    (amigo/amigo.cpp:323-402).  The device array ``self.vals`` is the
    authoritative copy; ``get_data()`` returns the host mirror.
    """

    def __init__(self, nrows, ncols, rowp, cols, vals=None, device=None,
                 diag_pos=None):
        """diag_pos: the position of each row's diagonal entry when the
        caller already knows it (otherwise found from the pattern)."""
        self.device = _device(device)
        self.nrows = int(nrows)
        self.ncols = int(ncols)
        self.rowp = np.ascontiguousarray(rowp, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.nnz = int(self.rowp[-1])
        self._host = None          # host mirror, made on first use
        if vals is not None:
            self.host_data[:] = np.asarray(vals, dtype=np.float64)
            self.vals = torch.from_numpy(self.host_data.copy()).to(self.device)
        else:
            self.vals = torch.zeros(self.nnz, dtype=torch.float64, device=self.device)
        self.d_rowp = torch.from_numpy(self.rowp).to(self.device)
        self.d_cols = torch.from_numpy(self.cols).to(self.device)
        if diag_pos is not None:
            self.diag = np.ascontiguousarray(diag_pos, dtype=np.int32)
            self.d_diag = torch.from_numpy(np.maximum(self.diag, 0)).to(self.device)
            return
        # first position of column i in row i, -1 when absent
        diag = np.full(self.nrows, -1, dtype=np.int64)
        rows = np.repeat(np.arange(self.nrows), np.diff(self.rowp))
        hit = np.nonzero(self.cols[: self.nnz] == rows)[0]
        if len(hit):
            r = rows[hit]
            first = np.ones(len(hit), bool)
            first[1:] = r[1:] != r[:-1]
            diag[r[first]] = hit[first]
        self.diag = diag.astype(np.int32)
        diag = self.diag
        self.d_diag = torch.from_numpy(np.maximum(diag, 0)).to(self.device)

    @property
    def host_data(self):
        if self._host is None:
            self._host = np.zeros(self.nnz)
        return self._host

    def get_nonzero_structure(self):
        return self.nrows, self.ncols, self.nnz, self.rowp, self.cols

    def get_data(self):
        return self.host_data

    def copy_data_device_to_host(self):
        self.host_data[:] = self.vals.cpu().numpy()

    def copy_data_host_to_device(self):
        self.vals.copy_(torch.from_numpy(self.host_data))

    def zero(self):
        self.vals.zero_()

    def add_diagonal(self, diag):
        """vals[diag_pos[i]] += diag[i] on the device (CSRMat::add_diagonal,
        include/csr_matrix.h:508-528).  ``diag`` is a device tensor, a Vector
        or a host array."""
        if np.any(self.diag < 0):
            raise ValueError("matrix pattern lacks a diagonal entry")
        d = diag.dev if isinstance(diag, Vector) else diag
        if not torch.is_tensor(d):
            d = torch.as_tensor(np.asarray(d, dtype=np.float64), device=self.device)
        d = d.to(self.device, torch.float64).contiguous()
        _lib.call("ab_csr_add_diagonal", self.nrows, self.d_diag.data_ptr(),
                  d.data_ptr(), self.vals.data_ptr(), _stream_ptr(self.device))

    def mult(self, x, y):
        """y = K x on the device; x, y are device tensors or Vectors."""
        xd = x.dev if isinstance(x, Vector) else x
        yd = y.dev if isinstance(y, Vector) else y
        _lib.call("ab_csr_matvec", self.nrows, self.d_rowp.data_ptr(),
                  self.d_cols.data_ptr(), self.vals.data_ptr(), xd.data_ptr(),
                  yd.data_ptr(), _stream_ptr(self.device))


class LdlTuning(ctypes.Structure):
    """ab_ldl_tuning (include/amigo_b200.h)."""
    _fields_ = [("panel_mode", ctypes.c_int), ("cl_min_rows", ctypes.c_int),
                ("panel_cache_bytes", ctypes.c_int),
                ("cluster_entries", ctypes.c_longlong),
                ("wide_entries", ctypes.c_longlong), ("solve_queue", ctypes.c_int),
                ("factor_ms", ctypes.c_double), ("solve_ms", ctypes.c_double),
                ("factor_ms_initial", ctypes.c_double),
                ("solve_ms_initial", ctypes.c_double),
                ("configurations", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# Settings found by the autotuner, per pattern and precision: a later
# handle of the same pattern takes them without timing again.
_TUNED = {}


def _pattern_key(rowps, colss, precision):
    import hashlib
    hsh = hashlib.blake2b(digest_size=16)
    for rp, cl in zip(rowps, colss):
        hsh.update(np.ascontiguousarray(rp, dtype=np.int32).tobytes())
        hsh.update(np.ascontiguousarray(cl, dtype=np.int32).tobytes())
    return (len(rowps), hsh.hexdigest(), precision)


def _autotune(h, vals, device, key, reps, cache):
    """ab_ldl_autotune on the handle (or the cached settings of its
    pattern, then one factorization); returns the settings as a dict with
    'cached' set accordingly."""
    t = LdlTuning()
    with torch.cuda.device(device):
        if cache and key in _TUNED:
            t = _TUNED[key]
            _lib.call("ab_ldl_apply_tuning", h, ctypes.byref(t))
            _lib.call("ab_ldl_factor", h, vals.data_ptr(), _stream_ptr(device))
            return dict(t.as_dict(), cached=True)
        _lib.call("ab_ldl_autotune", h, vals.data_ptr(), int(reps),
                  _stream_ptr(device), ctypes.byref(t))
    if cache:
        _TUNED[key] = t
    return dict(t.as_dict(), cached=False)


class SparseLDL:
    """amigo.SparseLDL on the GPU (include/sparse_ldl.h:20).

    ``SparseLDL(mat, solver_type=LDL, ustab=0.01, pivot_tol=1e-14,
    delay_growth=2.0, order=NATURAL)`` performs the symbolic analysis (host,
    bit-identical to the reference's) and uploads the device plan;
    ``factor()`` factors ``mat``'s current device values and returns 0;
    ``solve(x)`` overwrites x (a Vector, a device tensor, or a float64 numpy
    array of shape (n,) or (n, nrhs)); ``get_inertia()`` returns
    (npos, nneg).
    """

    def __init__(self, mat, solver_type=SolverType.LDL, ustab=0.01,
                 pivot_tol=1e-14, delay_growth=2.0,
                 order=OrderingType.NATURAL, precision="fp64"):
        if int(solver_type) != int(SolverType.LDL):
            raise NotImplementedError(
                "SolverType.CHOLESKY is not provided by amigo_b200")
        self.mat = mat
        self.n = mat.nrows
        self.device = mat.device
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("ab_ldl_create", self.n, _iptr(mat.rowp), _iptr(mat.cols),
                      int(order), int(solver_type), float(ustab),
                      float(pivot_tol), float(delay_growth), ctypes.byref(h))
        self._h = h
        self._factored = False
        self.precision = "fp64"
        if precision != "fp64":
            self.set_precision(precision)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().ab_ldl_destroy(h)
            except Exception:
                pass
            self._h = None

    def symbolic(self):
        return symbolic_arrays(self._h)

    def factor(self):
        with torch.cuda.device(self.device):
            _lib.call("ab_ldl_factor", self._h, self.mat.vals.data_ptr(),
                      _stream_ptr(self.device))
        self._factored = True
        self.factor_count = getattr(self, "factor_count", 0) + 1
        return 0

    def get_inertia(self):
        p, q = ctypes.c_int(), ctypes.c_int()
        _lib.call("ab_ldl_inertia", self._h, _stream_ptr(self.device),
                  ctypes.byref(p), ctypes.byref(q))
        return p.value, q.value

    def set_precision(self, precision):
        """Front precision of the next factorizations: "fp64" (default) or
        "fp32" (mixed precision: FP32 fronts, FP64 pivot tests and solve
        accumulation; pair with FP64 iterative refinement)."""
        bits = {"fp64": 64, "fp32": 32, 64: 64, 32: 32}[precision]
        _lib.call("ab_ldl_set_precision", self._h, bits)
        self.precision = "fp64" if bits == 64 else "fp32"

    def set_tensor_cores(self, on):
        """FP32 fronts: Schur updates of the large fronts on the tensor
        cores (3xTF32, default) or on the CUDA cores."""
        _lib.call("ab_ldl_set_tensor_cores", self._h, int(bool(on)))

    def set_panel_cache(self, nbytes):
        """Shared memory of the large-front panel kernel for a copy of the
        panel's L columns (0 .. 204800 bytes; default 0 reads them from
        HBM)."""
        _lib.call("ab_ldl_set_panel_cache", self._h, int(nbytes))

    def set_cluster_threshold(self, entries):
        """Fronts with f * npiv >= entries (below the wide threshold) are
        solved by a thread-block cluster of 8 CTAs each."""
        _lib.call("ab_ldl_set_cluster_threshold", self._h, int(entries))

    def set_solve_queue(self, mode):
        """Narrow-front solve schedule (ab_ldl_set_solve_queue): bit 0 one
        work-queue launch per sweep over the all-narrow levels, bit 1
        fronts of at most 128 rows on 128-thread CTAs; default 1; every
        mode gives the same result bit for bit."""
        _lib.call("ab_ldl_set_solve_queue", self._h, int(mode))

    def solve_status(self):
        """Raise if a work-queue solve sweep's wait ran out since the last
        check (ab_ldl_solve_status)."""
        _lib.call("ab_ldl_solve_status", self._h, _stream_ptr(self.device))

    def set_panel_mode(self, mode, min_rows=0):
        """Large-front panels: 0 (default) a thread-block cluster of 8 CTAs
        per front on levels whose largest front has >= min_rows rows (fronts
        past shared memory with W and L in global scratch, on clusters of 8
        or 16), 1 one CTA per front, 2 cluster panels with the one-CTA
        widths (identical results to mode 1), 3 the global-scratch form on
        clusters of 16 wherever it applies (identical results to mode 0)."""
        _lib.call("ab_ldl_set_panel_mode", self._h, int(mode), int(min_rows))

    def set_wide_threshold(self, entries):
        """Fronts with f * npiv >= entries are solved by the multi-CTA
        kernels (default 2^22)."""
        _lib.call("ab_ldl_set_wide_threshold", self._h, int(entries))

    def stats(self):
        fl, fe = ctypes.c_double(), ctypes.c_double()
        mf, nd, lv = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.call("ab_ldl_stats", self._h, _stream_ptr(self.device),
                  ctypes.byref(fl), ctypes.byref(fe), ctypes.byref(mf),
                  ctypes.byref(nd), ctypes.byref(lv))
        return dict(flops=fl.value, factor_entries=fe.value, max_front=mf.value,
                    num_delayed=nd.value, levels=lv.value)

    def node_pivots(self):
        nn = self.symbolic()["num_nodes"]
        a = np.zeros(nn, np.int32)
        b = np.zeros(nn, np.int32)
        _lib.call("ab_ldl_node_pivots", self._h, _stream_ptr(self.device),
                  _iptr(a), _iptr(b))
        return a, b

    def autotune(self, reps=3, cache=True):
        """Pick the large-front panel form and the solve schedule for this
        pattern by timing them on mat's current values
        (ab_ldl_autotune); the handle is left factored with the chosen
        settings.  Panel forms change the factorization only to rounding,
        the solve thresholds the solution only to rounding.  With
        `cache`, a later SparseLDL of the same pattern and precision takes
        the stored settings without timing.  Returns the settings and the
        best factor / solve times before and after (ms)."""
        key = _pattern_key([self.mat.rowp], [self.mat.cols], self.precision)
        out = _autotune(self._h, self.mat.vals, self.device, key, reps, cache)
        self._factored = True
        self.factor_count = getattr(self, "factor_count", 0) + 1
        return out

    def solve_device(self, xd):
        """Solve in place on a device tensor of shape (n,) or (nrhs, n)
        (rows contiguous: each right-hand side is one contiguous column of
        the column-major n x nrhs array)."""
        if xd.dtype != torch.float64 or not xd.is_cuda or not xd.is_contiguous():
            raise TypeError("expected a contiguous float64 CUDA tensor")
        nrhs = 1 if xd.dim() == 1 else xd.shape[0]
        with torch.cuda.device(self.device):
            _lib.call("ab_ldl_solve", self._h, xd.data_ptr(), nrhs, self.n,
                      _stream_ptr(self.device))

    def solve(self, x):
        if isinstance(x, Vector):
            self.solve_device(x.dev)
            return
        if torch.is_tensor(x):
            self.solve_device(x)
            return
        if isinstance(x, np.ndarray):
            if x.dtype != np.float64:
                raise TypeError("NumPy array must have dtype=float64")
            if x.ndim not in (1, 2):
                raise TypeError("NumPy array must be 1D or 2D")
            if not x.flags.writeable:
                raise TypeError("NumPy array must be writeable")
            cols = x.reshape(self.n, -1).T if x.ndim == 2 else x[None, :]
            xd = torch.from_numpy(np.ascontiguousarray(cols)).to(self.device)
            self.solve_device(xd if x.ndim == 2 else xd[0])
            out = xd.cpu().numpy()
            if x.ndim == 1:
                x[:] = out[0]
            else:
                x[:, :] = out.T
            return
        raise RuntimeError("Expected either a NumPy array or amigo_b200.Vector")


class SolveGraph:
    """A solve on one device buffer captured as a CUDA graph.

    ``g = SolveGraph(ldl, xd)``; ``g()`` solves in place on ``xd`` (as
    ``ldl.solve_device(xd)``, same bits) by replaying the graph on the
    current stream.  The solve's launch schedule depends on the front sizes
    of the factorization (delayed pivots), so the graph is captured again
    on the first call after each ``ldl.factor()``; replays between
    factorizations cost one graph launch instead of one launch per level
    and sweep.  The work-queue sweeps take their epoch from device memory,
    so every replay is a fresh sweep.  ``ab_launch_count`` counts the
    captured kernels once, at capture."""

    def __init__(self, ldl, xd):
        if xd.dtype != torch.float64 or not xd.is_cuda or not xd.is_contiguous():
            raise TypeError("expected a contiguous float64 CUDA tensor")
        self.ldl = ldl
        self.xd = xd
        self.graph = None
        self._count = None
        self.captures = 0
        self.replays = 0

    def _capture(self):
        ldl, xd = self.ldl, self.xd
        # the host-side schedule of this factorization is built by one solve
        # outside the capture (on a copy)
        warm = xd.clone()
        ldl.solve_device(warm)
        torch.cuda.current_stream(ldl.device).synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.device(ldl.device):
            with torch.cuda.graph(g):
                ldl.solve_device(xd)
        self.graph = g
        self._count = getattr(ldl, "factor_count", 0)
        self.captures += 1

    def __call__(self):
        if self.graph is None or self._count != getattr(self.ldl, "factor_count", 0):
            self.graph = None
            self._capture()
        self.graph.replay()
        self.replays += 1


def symbolic_arrays(h):
    nn, nc = ctypes.c_int(), ctypes.c_int()
    _lib.call("ab_ldl_symbolic_sizes", h, ctypes.byref(nn), ctypes.byref(nc))
    nn, nc = nn.value, nc.value
    cp = ctypes.c_int()
    out = {}
    # n is recovered from the node partition
    arrs = dict(node_ptr=np.zeros(nn + 1, np.int32))
    _lib.call("ab_ldl_symbolic_arrays", h, _iptr(arrs["node_ptr"]), None, None,
              None, None, None, None)
    n = int(arrs["node_ptr"][-1]) if nn > 0 else 0
    out = dict(
        node_ptr=arrs["node_ptr"],
        node_to_var=np.zeros(max(n, 1), np.int32),
        children_ptr=np.zeros(nn + 2, np.int32),
        children=np.zeros(max(nn, 1), np.int32),
        contrib_ptr=np.zeros(nn + 1, np.int32),
        contrib_rows=np.zeros(max(nc, 1), np.int32),
        invperm=np.zeros(max(n, 1), np.int32),
    )
    _lib.call("ab_ldl_symbolic_arrays", h, *[_iptr(out[k]) for k in (
        "node_ptr", "node_to_var", "children_ptr", "children", "contrib_ptr",
        "contrib_rows", "invperm")])
    out["node_to_var"] = out["node_to_var"][:n]
    out["invperm"] = out["invperm"][:n]
    out["children"] = out["children"][:nn]
    out["contrib_rows"] = out["contrib_rows"][:nc]
    out["num_nodes"] = nn
    del cp
    return out


def analyze(n, rowp, cols, order=OrderingType.AMD):
    """Host-only symbolic analysis (no GPU needed); returns the arrays of
    ``SparseLDL.symbolic()``."""
    rowp = np.ascontiguousarray(rowp, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    h = ctypes.c_void_p()
    _lib.call("ab_ldl_analyze", int(n), _iptr(rowp), _iptr(cols), int(order),
              ctypes.byref(h))
    try:
        return symbolic_arrays(h)
    finally:
        _lib.lib().ab_ldl_destroy(h)


def mem_estimate(n, rowp, cols, precision=64, delay_growth=2.0, nrhs=1,
                 order=OrderingType.AMD):
    """Device bytes a factorization of this pattern needs (ab_ldl_mem_estimate),
    from its symbolic analysis on the host."""
    rowp = np.ascontiguousarray(rowp, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    h = ctypes.c_void_p()
    _lib.call("ab_ldl_analyze", int(n), _iptr(rowp), _iptr(cols), int(order),
              ctypes.byref(h))
    try:
        out = ctypes.c_longlong()
        _lib.call("ab_ldl_mem_estimate", h, int(precision), float(delay_growth),
                  int(nrhs), ctypes.byref(out))
        return int(out.value)
    finally:
        _lib.lib().ab_ldl_destroy(h)


class BatchedSparseLDL:
    """Many independent SparseLDL problems factored and solved together:
    one launch per elimination-tree level covers the fronts of every
    problem.  `patterns` is a list of (n, rowp, cols); the values passed to
    factor() and the vectors passed to solve are the problems'
    concatenation (device tensors).  get_inertia() returns a list of
    (npos, nneg), one per problem."""

    def __init__(self, patterns, ustab=0.01, pivot_tol=1e-14,
                 delay_growth=2.0, order=OrderingType.AMD, device=None):
        self.device = _device(device)
        self.k = len(patterns)
        ns = np.array([int(p[0]) for p in patterns], dtype=np.int32)
        self._rowp = [np.ascontiguousarray(p[1], dtype=np.int32) for p in patterns]
        self._cols = [np.ascontiguousarray(p[2], dtype=np.int32) for p in patterns]
        RP = (ctypes.POINTER(ctypes.c_int) * self.k)(*[_iptr(a) for a in self._rowp])
        CP = (ctypes.POINTER(ctypes.c_int) * self.k)(*[_iptr(a) for a in self._cols])
        self.n_each = ns
        self.nnz_each = np.array([int(a[-1]) for a in self._rowp])
        self.var_off = np.concatenate([[0], np.cumsum(ns)])
        self.nnz_off = np.concatenate([[0], np.cumsum(self.nnz_each)])
        self.n = int(self.var_off[-1])
        self.nnz = int(self.nnz_off[-1])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("ab_ldl_batch_create", self.k, _iptr(ns), RP, CP, int(order),
                      0, float(ustab), float(pivot_tol), float(delay_growth),
                      ctypes.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().ab_ldl_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_precision(self, precision):
        """Front precision ("fp64" default, or "fp32" mixed)."""
        bits = {"fp64": 64, "fp32": 32, 64: 64, 32: 32}[precision]
        _lib.call("ab_ldl_set_precision", self._h, bits)
        self.precision = "fp64" if bits == 64 else "fp32"

    def set_tensor_cores(self, on):
        _lib.call("ab_ldl_set_tensor_cores", self._h, int(bool(on)))

    def factor(self, vals):
        if vals.numel() != self.nnz or vals.dtype != torch.float64:
            raise ValueError("expected the concatenated float64 values")
        with torch.cuda.device(self.device):
            _lib.call("ab_ldl_factor", self._h, vals.data_ptr(),
                      _stream_ptr(self.device))
        self.factor_count = getattr(self, "factor_count", 0) + 1
        return 0

    def autotune(self, vals, reps=3, cache=True):
        """See SparseLDL.autotune; `vals` are the concatenated values."""
        if vals.numel() != self.nnz or vals.dtype != torch.float64:
            raise ValueError("expected the concatenated float64 values")
        key = _pattern_key(self._rowp, self._cols, getattr(self, "precision", "fp64"))
        out = _autotune(self._h, vals, self.device, key, reps, cache)
        self.factor_count = getattr(self, "factor_count", 0) + 1
        return out

    def get_inertia(self):
        a = np.zeros(self.k, np.int32)
        b = np.zeros(self.k, np.int32)
        _lib.call("ab_ldl_batch_inertia", self._h, _stream_ptr(self.device),
                  _iptr(a), _iptr(b))
        return list(zip(a.tolist(), b.tolist()))

    def set_solve_queue(self, mode):
        """See SparseLDL.set_solve_queue."""
        _lib.call("ab_ldl_set_solve_queue", self._h, int(mode))

    def solve_status(self):
        _lib.call("ab_ldl_solve_status", self._h, _stream_ptr(self.device))

    def inertia_device(self):
        """Device pointer of the per-problem [npos, nneg] of the last
        factorization (ab_ldl_inertia_device)."""
        p = ctypes.c_void_p()
        _lib.call("ab_ldl_inertia_device", self._h, ctypes.byref(p))
        return p.value

    def solve_device(self, xd):
        nrhs = 1 if xd.dim() == 1 else xd.shape[0]
        with torch.cuda.device(self.device):
            _lib.call("ab_ldl_solve", self._h, xd.data_ptr(), nrhs, self.n,
                      _stream_ptr(self.device))

    def stats(self):
        fl, fe = ctypes.c_double(), ctypes.c_double()
        mf, nd, lv = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.call("ab_ldl_stats", self._h, _stream_ptr(self.device),
                  ctypes.byref(fl), ctypes.byref(fe), ctypes.byref(mf),
                  ctypes.byref(nd), ctypes.byref(lv))
        return dict(flops=fl.value, factor_entries=fe.value, max_front=mf.value,
                    num_delayed=nd.value, levels=lv.value)
