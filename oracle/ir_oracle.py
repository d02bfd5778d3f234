"""CPU restatement of amigo's iterative refinement on the unreduced 8-block
Newton system (test infrastructure only).

Follows DirectSparseSolver.iterative_refinement
(amigo/algorithm/solvers/linear_solver.py:109-264) step for step on numpy
arrays: K p via a CSR matvec, the four residual blocks, the ratio test
(stop below 1e-10 after >= 1 step, or when the ratio improves by less than
a factor 0.999999999), condensation, correction solve through `solve`, and
bound-dual back-substitution.  Pinned in tests against the reference's own
function run in this container.
"""
import numpy as np
import scipy.sparse as sp


def iterative_refinement(K, solve, mu, mult_ind, rhs_saved, g, zl, zu, sl, su,
                         lbx, ubx, px, max_steps=10):
    """Returns (px, dzl, dzu, steps_taken, last_ratio).  `solve(r)` returns
    K^{-1} r."""
    px = np.array(px, dtype=np.float64)
    n = len(px)
    pi = np.where(~mult_ind)[0]
    ci = np.where(mult_ind)[0]
    fl = np.isfinite(lbx)
    fu = np.isfinite(ubx)
    gl = np.where(fl, sl, 1.0)
    gu = np.where(fu, su, 1.0)
    sigma = np.where(fl, zl / gl, 0.0) + np.where(fu, zu / gu, 0.0)
    dx = px[pi]
    dzl = np.where(fl, (mu - gl * zl - zl * dx) / gl, 0.0)
    dzu = np.where(fu, (mu - gu * zu + zu * dx) / gu, 0.0)
    rhs_x = -(g[pi] - zl + zu)
    rhs_c = rhs_saved[ci]
    rhs_zl = np.where(fl, mu - gl * zl, 0.0)
    rhs_zu = np.where(fu, mu - gu * zu, 0.0)

    def amax(a):
        return np.max(np.abs(a)) if len(a) > 0 else 0.0

    nrm_rhs = max(amax(rhs_x), amax(rhs_c), amax(rhs_zl), amax(rhs_zu))
    ratio_old = 1e30
    ratio = None
    steps = 0
    for step in range(max_steps):
        Kpx = K @ px
        e_x = rhs_x - Kpx[pi] + sigma * dx + dzl - dzu
        e_c = rhs_c - Kpx[ci]
        e_zl = np.where(fl, rhs_zl - zl * dx - gl * dzl, 0.0)
        e_zu = np.where(fu, rhs_zu + zu * dx - gu * dzu, 0.0)
        nrm_resid = max(amax(e_x), amax(e_c), amax(e_zl), amax(e_zu))
        nrm_res = max(amax(px), amax(dzl), amax(dzu))
        ratio = nrm_resid / (min(nrm_res, 1e6 * nrm_rhs) + nrm_rhs)
        if ratio < 1e-10 and step >= 1:
            break
        if step >= 1 and ratio > 0.999999999 * ratio_old:
            break
        ratio_old = ratio
        e_cond = np.zeros(n)
        e_cond[pi] = e_x + np.where(fl, e_zl / gl, 0.0) - np.where(fu, e_zu / gu, 0.0)
        e_cond[ci] = e_c
        corr = solve(e_cond)
        dc = corr[pi]
        dzl = dzl + np.where(fl, (e_zl - zl * dc) / gl, 0.0)
        dzu = dzu + np.where(fu, (e_zu + zu * dc) / gu, 0.0)
        px = px + corr
        dx = px[pi]
        steps += 1
    return px, dzl, dzu, steps, ratio


def as_csr(vals, rowp, cols, n):
    return sp.csr_matrix((vals, cols, rowp), shape=(n, n))
