"""CPU restatement of the SIMP full-space models' Lagrangian, gradient and
Hessian (test infrastructure only; numpy).  The same functions serve the 2D
quad model (problems/simp2d.py) and the 3D hexahedron model
(problems/simp3d.py): the element sizes come from the model's K0 (ND x ND)
and filter matrix A (NV x NV).

The reference ships no component code for this exact model (its
generated per-component derivatives come from the absent A2D library, see
amigo/component.py:1022-1108), so this restatement is pinned by
finite differences of `lagrangian` in the tests rather than by reference
outputs: parity of the device element kernels against it is "parity
unpinned" with respect to the reference itself.
"""
import numpy as np


def _stiffness(m, r):
    from amigo_b200.problems.simp2d import E0, EMIN, PENALTY as p
    E = EMIN + r ** p * (E0 - EMIN)
    dE = p * r ** (p - 1) * (E0 - EMIN)
    d2E = p * (p - 1) * r ** (p - 2) * (E0 - EMIN)
    return E, dE, d2E


def _sizes(m):
    nd, nv = m.K0.shape[0], m.A.shape[0]
    return nd, nv, nd // nv


def _split(m, x):
    nd, nv, _ = _sizes(m)
    return (x[m.ev[:, :nd]], x[m.ev[:, nd:nd + nv]], x[m.ev[:, nd + nv:]],
            x[m.re0:m.re0 + m.nelems], x[m.fv[:, nv + 1:]])


def lagrangian(m, x, alpha=1.0):
    nd, nv, dim = _sizes(m)
    u, rt, lam, re, mu = _split(m, x)
    E, _, _ = _stiffness(m, rt.mean(axis=1))
    Ku = u @ m.K0.T
    L = alpha * (m.f @ x)                    # f^T u (f only has u entries)
    L += np.sum(E * np.sum(lam * Ku, axis=1))
    L -= x[m.lam0:m.lam0 + dim * m.nnodes] @ m.f[m.u0:m.u0 + dim * m.nnodes]
    L += np.sum(mu * (rt @ m.A.T)) - np.sum(mu.sum(axis=1) * re) / nv
    L += x[m.nu0] * (re.sum() / m.nelems - m.volfrac - x[m.s0])
    return L


def gradient(m, x, alpha=1.0):
    nd, nv, dim = _sizes(m)
    g = np.zeros(m.n)
    u, rt, lam, re, mu = _split(m, x)
    E, dE, _ = _stiffness(m, rt.mean(axis=1))
    Ku = u @ m.K0.T
    Kl = lam @ m.K0.T
    lKu = np.sum(lam * Ku, axis=1)
    np.add.at(g, m.ev[:, :nd], E[:, None] * Kl)
    np.add.at(g, m.ev[:, nd:nd + nv], (dE * lKu)[:, None] / nv + mu @ m.A)
    np.add.at(g, m.ev[:, nd + nv:], E[:, None] * Ku)
    np.add.at(g, m.fv[:, nv], -mu.sum(axis=1) / nv + x[m.nu0] / m.nelems)
    np.add.at(g, m.fv[:, nv + 1:], rt @ m.A.T - re[:, None] / nv)
    fu = m.f[m.u0:m.u0 + dim * m.nnodes]
    g[m.u0:m.u0 + dim * m.nnodes] += alpha * fu
    g[m.lam0:m.lam0 + dim * m.nnodes] -= fu
    g[m.nu0] += re.sum() / m.nelems - m.volfrac - x[m.s0]
    g[m.s0] += -x[m.nu0]
    return g


def hessian_dense_blocks(m, x):
    """Per-element (2 ND + NV)^2 elasticity and (2 NV + 1)^2 filter blocks."""
    nd, nv, _ = _sizes(m)
    u, rt, lam, _, _ = _split(m, x)
    E, dE, d2E = _stiffness(m, rt.mean(axis=1))
    Ku = u @ m.K0.T
    Kl = lam @ m.K0.T
    lKu = np.sum(lam * Ku, axis=1)
    ne, k = m.nelems, 2 * nd + nv
    R, L = slice(nd, nd + nv), slice(nd + nv, k)
    H = np.zeros((ne, k, k))
    H[:, :nd, R] = (dE[:, None] * Kl)[:, :, None] / nv
    H[:, R, :nd] = np.transpose(H[:, :nd, R], (0, 2, 1))
    H[:, :nd, L] = E[:, None, None] * m.K0[None]
    H[:, L, :nd] = E[:, None, None] * m.K0.T[None]
    H[:, R, R] = (d2E * lKu)[:, None, None] / (nv * nv)
    H[:, L, R] = (dE[:, None] * Ku)[:, :, None] / nv
    H[:, R, L] = np.transpose(H[:, L, R], (0, 2, 1))
    Fb = np.zeros((2 * nv + 1, 2 * nv + 1))
    Fb[nv + 1:, :nv] = m.A
    Fb[:nv, nv + 1:] = m.A.T
    Fb[nv + 1:, nv] = -1.0 / nv
    Fb[nv, nv + 1:] = -1.0 / nv
    return H, Fb


def hessian_values(m, x, alpha=1.0):
    """KKT values on m's CSR pattern, fixed rows/columns applied."""
    vals = np.zeros(m.nnz)
    H, Fb = hessian_dense_blocks(m, x)
    np.add.at(vals, m.epos.ravel(), H.reshape(-1))
    np.add.at(vals, m.fpos.ravel(), np.broadcast_to(Fb.ravel(), (m.nelems, Fb.size)).ravel())
    np.add.at(vals, m.vpos.ravel(), 1.0 / m.nelems)
    np.add.at(vals, m.spos, -1.0)
    vals[m.fixed_zero_pos] = 0.0
    vals[m.fixed_diag_pos] = 1.0
    return vals


def gradient_fixed(m, x, alpha=1.0):
    g = gradient(m, x, alpha)
    g[m.fixed] = 0.0
    return g
