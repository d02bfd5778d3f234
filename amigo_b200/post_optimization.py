"""Model outputs and post-optimality sensitivities on the resident factor.

`PostOptimization(optimizer, model)` is amigo's PostOptimization
(amigo/algorithm/post_optimization.py:13-77) for a generated model
(codegen.GeneratedModel) after `Optimizer.optimize()`:
  * compute_output(): the outputs every component instance declares
    (Component.add_output), concatenated group by group, instance by
    instance;
  * compute_post_opt_derivatives(of, wrt, method): d output / d data at the
    optimum, where `of` indexes the output vector and `wrt` the data vector
    (every group's E x ND data array, row-major, concatenated).  The KKT
    matrix at the optimum (Hessian plus the barrier diagonal, factored by
    the optimizer's linear solver with its objective scale and Hessian
    scaling, as the reference does) is solved once per output (adjoint,
    K lambda = -d out_i / dx; df/dd = d out/dd + (d g/dd)^T lambda) or once
    per data entry (direct, K dx = -d g / dd_j; df/dd_j = d out/dd_j +
    d out/dx dx).  On B200Solver all right-hand sides go to the device
    factor in one multi-right-hand-side solve.
The per-instance blocks of d out/dx, d out/dd and d(grad L)/dd come from the
generated `<group>_sens` evaluators (host build), assembled into sparse
matrices.
"""
import ctypes

import numpy as np
import scipy.sparse as sp

try:
    import torch
except ImportError:
    torch = None


def _arr(v):
    if torch is not None and isinstance(v, torch.Tensor):
        return v
    if hasattr(v, "dev"):
        return v.dev
    if hasattr(v, "arr"):
        return v.arr
    return v.get_array()


def _host(a):
    if torch is not None and isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


class PostOptimization:
    def __init__(self, optimizer, model):
        from .codegen import emit
        from .codegen.model import compile_module
        self.opt = optimizer
        self.model = model
        src = emit.module_source(list(zip(model.syms, [g.comp for g in model.groups])))
        self._lib = ctypes.CDLL(compile_module(src, host=True))
        self.num_outputs = sum(g.E * g.comp.num_outputs for g in model.groups)
        self.num_data = sum(g.E * g.comp.num_data for g in model.groups)

    # -- per-instance blocks -----------------------------------------------------
    def _blocks(self, x, alpha):
        P = ctypes.POINTER(ctypes.c_double)
        I = ctypes.POINTER(ctypes.c_int)
        x = np.ascontiguousarray(x, dtype=np.float64)
        out, rows = [], dict(oq=[], od=[], gd=[])
        o_off = d_off = 0
        for sym, gr in zip(self.model.syms, self.model.groups):
            nq, nd, no = gr.comp.num_vars, gr.comp.num_data, gr.comp.num_outputs
            E = gr.E
            o = np.zeros((E, max(no, 1)))
            dgd = np.zeros((E, nq, max(nd, 1)))
            doq = np.zeros((E, max(no, 1), nq))
            dod = np.zeros((E, max(no, 1), max(nd, 1)))
            data = np.ascontiguousarray(gr.data if nd else np.zeros((E, 1)))
            fn = getattr(self._lib, sym + "_sens_batch")
            fn(ctypes.c_int(E), gr.idx.ctypes.data_as(I), x.ctypes.data_as(P),
               data.ctypes.data_as(P), ctypes.c_double(alpha), o.ctypes.data_as(P),
               dgd.ctypes.data_as(P), doq.ctypes.data_as(P), dod.ctypes.data_as(P))
            orow = o_off + np.arange(E * no).reshape(E, no)
            dcol = d_off + np.arange(E * nd).reshape(E, nd)
            if no:
                out.append(o[:, :no].ravel())
                rows["oq"].append((np.repeat(orow, nq, axis=1).ravel(),
                                   np.tile(gr.idx, (1, no)).ravel(),
                                   doq[:, :no, :].ravel()))
            if no and nd:
                rows["od"].append((np.repeat(orow, nd, axis=1).ravel(),
                                   np.tile(dcol, (1, no)).ravel(),
                                   dod[:, :no, :nd].ravel()))
            if nd:
                rows["gd"].append((np.repeat(gr.idx, nd, axis=1).ravel(),
                                   np.tile(dcol, (1, nq)).ravel(),
                                   dgd[:, :, :nd].ravel()))
            o_off += E * no
            d_off += E * nd
        n, no, nd = self.model.n, self.num_outputs, self.num_data

        def mat(parts, shape):
            if not parts:
                return sp.csr_matrix(shape)
            r = np.concatenate([p[0] for p in parts])
            c = np.concatenate([p[1] for p in parts])
            v = np.concatenate([p[2] for p in parts])
            return sp.csr_matrix((v, (r, c)), shape=shape)

        outv = np.concatenate(out) if out else np.zeros(0)
        oq = mat(rows["oq"], (no, n))
        od = mat(rows["od"], (no, nd))
        gd = mat(rows["gd"], (n, nd)).tolil()
        # fixed variables have no gradient (their rows are identity rows)
        gd[self.model.fixed, :] = 0.0
        return outv, oq, od, gd.tocsr()

    def compute_output(self):
        x = _host(_arr(self.opt.vars.get_solution()))
        return self._blocks(x, self.opt.obj_scale)[0]

    # -- solves on the factor at the optimum ----------------------------------------
    def _factor(self):
        o = self.opt
        x = o.vars.get_solution()
        o.ipo.compute_diagonal(o.vars, o.diag)
        if hasattr(o.diag, "copy_host_to_device") and not hasattr(o.diag, "dev"):
            o.diag.copy_host_to_device()
        o.solver.factor(o.obj_scale, x, o.diag, post_hessian=o.scale_fn)

    def _solve_many(self, R):
        """Rows of R (m x n, host) solved with the factor: one device
        multi-right-hand-side solve on B200Solver, else one solve each."""
        o = self.opt
        S = o.solver
        if hasattr(S, "ldl") and hasattr(S.ldl, "solve_device") and torch is not None:
            X = torch.from_numpy(np.ascontiguousarray(R, dtype=np.float64)).to(S.device)
            if X.shape[0]:
                S.ldl.solve_device(X if X.shape[0] > 1 else X[0])
            return X.cpu().numpy().reshape(R.shape)
        out = np.zeros_like(R)
        res, px = o.res, o.px
        for i in range(R.shape[0]):
            a = _arr(res)
            a[...] = R[i] if not (torch is not None and isinstance(a, torch.Tensor)) \
                else torch.from_numpy(R[i]).to(a.device)
            if hasattr(res, "copy_host_to_device") and not hasattr(res, "dev"):
                res.copy_host_to_device()
            S.solve(res, px)
            out[i] = _host(_arr(px))
        return out

    def compute_post_opt_derivatives(self, of=(), wrt=(), method="adjoint"):
        """d outputs[of] / d data[wrt] at the optimum (len(of) x len(wrt));
        method "adjoint" (one solve per output) or "direct" (one per data
        entry), as amigo's compute_post_opt_derivatives."""
        of = np.asarray(of, dtype=np.int64)
        wrt = np.asarray(wrt, dtype=np.int64)
        x = _host(_arr(self.opt.vars.get_solution()))
        _, oq, od, gd = self._blocks(x, self.opt.obj_scale)
        self._factor()
        dfdx = np.zeros((len(of), len(wrt)))
        if method == "adjoint":
            lam = self._solve_many(-oq[of, :].toarray())
            adj = (gd.T @ lam.T).T            # len(of) x n_data
            dfdx[:] = od[of][:, wrt].toarray() + adj[:, wrt]
        elif method == "direct":
            dx = self._solve_many(-gd[:, wrt].toarray().T)
            dirx = oq @ dx.T                  # n_out x len(wrt)
            dfdx[:] = od[of][:, wrt].toarray() + dirx[of, :]
        else:
            raise ValueError("method must be 'adjoint' or 'direct'")
        return dfdx
