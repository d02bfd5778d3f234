"""Device-side models for the component evaluation kernels (fem_simp.cu,
cartpole.cu)."""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import Simp2DStruct, Simp3DStruct
from .linalg import _stream_ptr


class SimpDevice:
    """Uploads a SIMP model's (problems.simp2d.Simp2D or
    problems.simp3d.Simp3D) index maps and constants."""

    dim = 2
    _struct = Simp2DStruct
    _prefix = "ab_simp2d"

    def __init__(self, model, device):
        from .problems import simp2d as S
        self.model = model
        self.device = torch.device(device)
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(self.device)
        colors = model.color_lists()
        cptr = np.cumsum([0] + [len(c) for c in colors])
        nu = self.dim * model.nnodes
        fu = model.f[model.u0:model.u0 + nu]
        li = np.nonzero(fu)[0]
        self._keep = dict(
            color_elems=t(np.concatenate(colors), np.int32),
            ev=t(model.ev, np.int32), fv=t(model.fv, np.int32),
            epos=t(model.epos, np.int32), fpos=t(model.fpos, np.int32),
            vpos=t(model.vpos, np.int32), spos=t(model.spos, np.int32),
            fixed=t(model.fixed, np.int32),
            fixed_zero_pos=t(model.fixed_zero_pos, np.int32),
            fixed_diag_pos=t(model.fixed_diag_pos, np.int32),
            load_idx=t(li, np.int32), load_val=t(fu[li], np.float64),
            K0=t(model.K0, np.float64), A=t(model.A, np.float64),
        )
        k = self._keep
        st = self._struct()
        st.n, st.nnz, st.nelems, st.nnodes = model.n, model.nnz, model.nelems, model.nnodes
        st.u0, st.rt0, st.re0, st.s_index = model.u0, model.rt0, model.re0, model.s0
        st.lam0, st.mu0, st.nu_index = model.lam0, model.mu0, model.nu0
        for i in range(len(cptr)):
            st.color_ptr[i] = int(cptr[i])
        for name in ("color_elems", "ev", "fv", "epos", "fpos", "vpos", "spos",
                     "fixed", "fixed_zero_pos", "fixed_diag_pos", "load_idx",
                     "load_val", "K0", "A"):
            setattr(st, name, k[name].data_ptr())
        st.nfixed = len(model.fixed)
        st.nfixed_zero = len(model.fixed_zero_pos)
        st.nload = int(k["load_idx"].numel())
        st.Bq = 1.0 / model.conn.shape[1]      # element volume / nodes
        st.vcoef = 1.0 / model.nelems
        st.volfrac = model.volfrac
        st.E0, st.Emin, st.penalty = S.E0, S.EMIN, S.PENALTY
        self.st = st

    def gradient(self, x, alpha, grad):
        _lib.call(self._prefix + "_gradient", ctypes.byref(self.st), x.data_ptr(),
                  float(alpha), grad.data_ptr(), _stream_ptr(self.device))

    def hessian(self, x, alpha, vals):
        _lib.call(self._prefix + "_hessian", ctypes.byref(self.st), x.data_ptr(),
                  float(alpha), vals.data_ptr(), _stream_ptr(self.device))


class Simp2DDevice(SimpDevice):
    pass


class Simp3DDevice(SimpDevice):
    dim = 3
    _struct = Simp3DStruct
    _prefix = "ab_simp3d"


class CartPoleDevice:
    """Uploads a problems.cartpole.CartPole model's (or CartPoleBatch's)
    index maps and constants."""

    def __init__(self, model, device, batch=False):
        from ._lib import CartPoleStruct
        from .problems import cartpole as C
        self.model = model
        self.device = torch.device(device)
        ti = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(self.device)
        td = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)
        self._keep = dict(iv=ti(model.iv), ipos=ti(model.ipos), bv=ti(model.bv),
                          bpos=ti(model.bpos))
        st = CartPoleStruct()
        st.n, st.nnz, st.N = model.n, model.nnz, model.N
        st.M, st.l, st.g = C.M_CART, C.L_POLE, C.GRAV
        if batch:
            self._keep.update(h_iv=td(model.h_iv), m_iv=td(model.m_iv),
                              inst_iv=ti(model.inst_iv))
            st.h, st.m = 0.0, 0.0
            st.nbc = 2 * model.k
            st.ninst = model.k
            self.ninst = model.k
        else:
            st.h, st.m = model.h, model.m_pole
            self.ninst = 1
        for k, v in self._keep.items():
            setattr(st, k, v.data_ptr())
        self.st = st

    def gradient(self, x, alpha, grad):
        _lib.call("ab_cartpole_gradient", ctypes.byref(self.st), x.data_ptr(),
                  float(alpha), grad.data_ptr(), _stream_ptr(self.device))

    def hessian(self, x, alpha, vals):
        _lib.call("ab_cartpole_hessian", ctypes.byref(self.st), x.data_ptr(),
                  float(alpha), vals.data_ptr(), _stream_ptr(self.device))

    def objective(self, x, out):
        """Objective value(s) into out[0] (or out[b] per instance)."""
        _lib.call("ab_cartpole_objective", ctypes.byref(self.st), x.data_ptr(),
                  out.data_ptr(), _stream_ptr(self.device))
