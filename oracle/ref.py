"""ctypes access to the reference's own CPU code (oracle/_ref/libamigo_ref.so).

Test infrastructure only: this module is imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the
product package.  The library is built by oracle/build_ref.sh from the
reference's header-only sources (include/sparse_ldl.h, include/block_amd.h,
include/ordering_utils.h, include/interior_point_backend.h).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libamigo_ref.so")

# OrderingType values in the reference (include/ordering_utils.h:21).
ORDER = {"NESTED_DISSECTION": 0, "AMD": 1, "MULTI_COLOR": 2, "NATURAL": 3}

_lib = None

_i = ctypes.c_int
_d = ctypes.c_double
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(
                "reference oracle library missing: run oracle/build_ref.sh "
                "(needs the reference sources)")
        L = ctypes.CDLL(LIB_PATH)
        L.ref_ldl_create.restype = _vp
        L.ref_ldl_create.argtypes = [_i, _ip, _ip, _i, _d, _d, _d, _i]
        L.ref_ldl_destroy.argtypes = [_vp]
        L.ref_ldl_num_nodes.argtypes = [_vp]
        L.ref_ldl_contrib_total.argtypes = [_vp]
        L.ref_ldl_symbolic.argtypes = [_vp, _ip, _ip, _ip, _ip, _ip, _ip, _ip]
        L.ref_ldl_set_values.argtypes = [_vp, _dp]
        L.ref_ldl_factor.argtypes = [_vp]
        L.ref_ldl_inertia.argtypes = [_vp, _ip, _ip]
        L.ref_ldl_solve.argtypes = [_vp, _i, _dp, _i]
        L.ref_ldl_node_pivots.argtypes = [_vp, _ip, _ip]
        L.ref_order.argtypes = [_i, _ip, _ip, _i, _ip, _ip]
        L.ref_set_blas_threads.argtypes = [_i]
        L.ref_set_blas_threads(1)
        for name in ("ref_ipm_compute_barrier_log_sum",
                     "ref_ipm_compute_barrier_dphi",
                     "ref_ipm_compute_constraint_violation_1norm"):
            getattr(L, name).restype = _d
        _lib = L
    return _lib


def set_blas_threads(n):
    """OpenBLAS threads used inside the reference's BLAS/LAPACK calls."""
    lib().ref_set_blas_threads(int(n))


def _ptr(a, kind):
    return a.ctypes.data_as(_ip if kind == "i" else _dp)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class RefSparseLDL:
    """The reference SparseLDL (include/sparse_ldl.h:20) on a CSR pattern."""

    def __init__(self, n, rowp, cols, order="AMD", ustab=0.01,
                 pivot_tol=1e-14, delay_growth=2.0, cholesky=False):
        self.n = int(n)
        self.rowp = _i32(rowp)
        self.cols = _i32(cols)
        self.nnz = int(self.rowp[-1])
        self._h = lib().ref_ldl_create(
            self.n, _ptr(self.rowp, "i"), _ptr(self.cols, "i"),
            ORDER[order] if isinstance(order, str) else int(order),
            ustab, pivot_tol, delay_growth, 1 if cholesky else 0)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ref_ldl_destroy(self._h)
            self._h = None

    def symbolic(self):
        L = lib()
        nn = L.ref_ldl_num_nodes(self._h)
        nc = L.ref_ldl_contrib_total(self._h)
        out = dict(
            node_ptr=np.zeros(nn + 1, np.int32),
            node_to_var=np.zeros(self.n, np.int32),
            children_ptr=np.zeros(nn + 2, np.int32),
            children=np.zeros(max(nn, 1), np.int32),
            contrib_ptr=np.zeros(nn + 1, np.int32),
            contrib_rows=np.zeros(max(nc, 1), np.int32),
            invperm=np.zeros(self.n, np.int32),
        )
        L.ref_ldl_symbolic(self._h, *[_ptr(out[k], "i") for k in (
            "node_ptr", "node_to_var", "children_ptr", "children",
            "contrib_ptr", "contrib_rows", "invperm")])
        out["children"] = out["children"][:nn]
        out["contrib_rows"] = out["contrib_rows"][:nc]
        out["num_nodes"] = nn
        return out

    def factor(self, vals):
        v = _f64(vals)
        assert v.shape[0] == self.nnz
        L = lib()
        L.ref_ldl_set_values(self._h, _ptr(v, "d"))
        return L.ref_ldl_factor(self._h)

    def inertia(self):
        p, q = ctypes.c_int(0), ctypes.c_int(0)
        lib().ref_ldl_inertia(self._h, ctypes.byref(p), ctypes.byref(q))
        return p.value, q.value

    def node_pivots(self):
        nn = lib().ref_ldl_num_nodes(self._h)
        npiv = np.zeros(nn, np.int32)
        ndel = np.zeros(nn, np.int32)
        lib().ref_ldl_node_pivots(self._h, _ptr(npiv, "i"), _ptr(ndel, "i"))
        return npiv, ndel

    def solve(self, b):
        b = np.array(b, dtype=np.float64, order="F", copy=True)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        lib().ref_ldl_solve(self._h, nrhs, _ptr(b, "d"), self.n)
        return b


def order(n, rowp, cols, kind="AMD"):
    """Reference OrderingUtils::copy_for_reorder + reorder
    (include/ordering_utils.h:38-56, 313-360)."""
    rowp = _i32(rowp)
    cols = _i32(cols)
    perm = np.zeros(n, np.int32)
    iperm = np.zeros(n, np.int32)
    lib().ref_order(n, _ptr(rowp, "i"), _ptr(cols, "i"), ORDER[kind],
                    _ptr(perm, "i"), _ptr(iperm, "i"))
    return perm, iperm


class RefIPM:
    """The reference's IPM vector functions (include/interior_point_backend.h)
    on numpy arrays; `info` holds pidx, cidx, lbx, ubx, lbh."""

    def __init__(self, pidx, cidx, lbx, ubx, lbh):
        self.pidx = _i32(pidx)
        self.cidx = _i32(cidx)
        self.lbx = _f64(lbx)
        self.ubx = _f64(ubx)
        self.lbh = _f64(lbh)

    def _args(self, xlam, zl, zu, sl, su):
        self._keep = [_f64(a) for a in (xlam, zl, zu, sl, su)]
        return [len(self.pidx), len(self.cidx), _ptr(self.pidx, "i"),
                _ptr(self.cidx, "i"), _ptr(self.lbx, "d"), _ptr(self.ubx, "d"),
                _ptr(self.lbh, "d")] + [_ptr(a, "d") for a in self._keep]

    def compute_residual(self, mu, st, grad):
        g = _f64(grad)
        res = np.zeros_like(g)
        lib().ref_ipm_compute_residual(_d(mu), *self._args(*st), _ptr(g, "d"),
                                       _ptr(res, "d"))
        return res

    def compute_diagonal(self, st, n):
        diag = np.zeros(n)
        lib().ref_ipm_compute_diagonal(*self._args(*st), _ptr(diag, "d"))
        return diag

    def compute_bound_dual_step(self, mu, st, px):
        px = _f64(px)
        dzl = np.zeros(len(self.pidx))
        dzu = np.zeros(len(self.pidx))
        lib().ref_ipm_compute_bound_dual_step(
            _d(mu), *self._args(*st), _ptr(px, "d"), _ptr(dzl, "d"),
            _ptr(dzu, "d"))
        return dzl, dzu

    def compute_max_step(self, tau, st, px, dzl, dzu):
        px, dzl, dzu = _f64(px), _f64(dzl), _f64(dzu)
        ax, az = ctypes.c_double(1.0), ctypes.c_double(1.0)
        xi, zi = ctypes.c_int(-1), ctypes.c_int(-1)
        lib().ref_ipm_compute_max_step(
            _d(tau), *self._args(*st), _ptr(px, "d"), _ptr(dzl, "d"),
            _ptr(dzu, "d"), ctypes.byref(ax), ctypes.byref(xi),
            ctypes.byref(az), ctypes.byref(zi))
        return ax.value, xi.value, az.value, zi.value

    def apply_step(self, ax, az, st, dxlam, dzl, dzu):
        xlam, zl, zu, sl, su = [np.array(a, dtype=np.float64) for a in st]
        dxlam, dzl, dzu = _f64(dxlam), _f64(dzl), _f64(dzu)
        out = [xlam.copy(), zl.copy(), zu.copy(), sl.copy(), su.copy()]
        lib().ref_ipm_apply_step(
            _d(ax), _d(az), *self._args(*st), _ptr(dxlam, "d"), _ptr(dzl, "d"),
            _ptr(dzu, "d"), _ptr(out[0], "d"), len(xlam), _ptr(out[1], "d"),
            _ptr(out[2], "d"), _ptr(out[3], "d"), _ptr(out[4], "d"))
        return out

    def compute_complementarity(self, st):
        part = np.zeros(2)
        mn = ctypes.c_double(np.inf)
        lib().ref_ipm_compute_complementarity(*self._args(*st), _ptr(part, "d"),
                                              ctypes.byref(mn))
        return part[0], part[1], mn.value

    def compute_kkt_error(self, mu, st, grad):
        g = _f64(grad)
        d, p, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lib().ref_ipm_compute_kkt_error(_d(mu), *self._args(*st), _ptr(g, "d"),
                                        ctypes.byref(d), ctypes.byref(p),
                                        ctypes.byref(c))
        return d.value, p.value, c.value

    def compute_barrier_log_sum(self, mu, st):
        return lib().ref_ipm_compute_barrier_log_sum(_d(mu), *self._args(*st))

    def compute_barrier_dphi(self, mu, st, grad, px):
        g, px = _f64(grad), _f64(px)
        return lib().ref_ipm_compute_barrier_dphi(_d(mu), *self._args(*st),
                                                  _ptr(g, "d"), _ptr(px, "d"))

    def reset_bound_multipliers(self, mu, kappa, st):
        zl = np.array(st[1], dtype=np.float64)
        zu = np.array(st[2], dtype=np.float64)
        lib().ref_ipm_reset_bound_multipliers(
            _d(mu), _d(kappa), *self._args(*st), _ptr(zl, "d"), _ptr(zu, "d"))
        return zl, zu

    def compute_affine_start_point(self, beta_min, st, dzl, dzu):
        dzl, dzu = _f64(dzl), _f64(dzu)
        zl = np.array(st[1], dtype=np.float64)
        zu = np.array(st[2], dtype=np.float64)
        lib().ref_ipm_compute_affine_start_point(
            _d(beta_min), *self._args(*st), _ptr(dzl, "d"), _ptr(dzu, "d"),
            _ptr(zl, "d"), _ptr(zu, "d"))
        return zl, zu

    def compute_max_comp_deviation(self, st, mu):
        md = ctypes.c_double()
        lib().ref_ipm_compute_max_comp_deviation(*self._args(*st), _d(mu),
                                                 ctypes.byref(md))
        return md.value

    def compute_complementarity_sq(self, st, mu):
        sq = ctypes.c_double()
        lib().ref_ipm_compute_complementarity_sq(*self._args(*st), _d(mu),
                                                 ctypes.byref(sq))
        return sq.value

    def compute_constraint_violation_1norm(self, st, grad):
        g = _f64(grad)
        return lib().ref_ipm_compute_constraint_violation_1norm(
            *self._args(*st), _ptr(g, "d"))
