"""CPU restatement of the 2D SIMP full-space model's Lagrangian, gradient
and Hessian (test infrastructure only; numpy).

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


def lagrangian(m, x, alpha=1.0):
    u = x[m.ev[:, :8]]
    rt = x[m.ev[:, 8:12]]
    lam = x[m.ev[:, 12:]]
    re = x[m.re0:m.re0 + m.nelems]
    mu = x[m.fv[:, 5:]]
    E, _, _ = _stiffness(m, rt.mean(axis=1))
    Ku = u @ m.K0.T
    L = alpha * (m.f @ x)                    # f^T u (f only has u entries)
    L += np.sum(E * np.sum(lam * Ku, axis=1))
    L -= x[m.lam0:m.lam0 + 2 * m.nnodes] @ m.f[m.u0:m.u0 + 2 * m.nnodes]
    L += np.sum(mu * (rt @ m.A.T)) - 0.25 * np.sum(mu.sum(axis=1) * re)
    L += x[m.nu0] * (re.sum() / m.nelems - m.volfrac - x[m.s0])
    return L


def gradient(m, x, alpha=1.0):
    g = np.zeros(m.n)
    u = x[m.ev[:, :8]]
    rt = x[m.ev[:, 8:12]]
    lam = x[m.ev[:, 12:]]
    re = x[m.re0:m.re0 + m.nelems]
    mu = x[m.fv[:, 5:]]
    E, dE, _ = _stiffness(m, rt.mean(axis=1))
    Ku = u @ m.K0.T
    Kl = lam @ m.K0.T
    lKu = np.sum(lam * Ku, axis=1)
    np.add.at(g, m.ev[:, :8], E[:, None] * Kl)
    np.add.at(g, m.ev[:, 8:12], 0.25 * (dE * lKu)[:, None] + mu @ m.A)
    np.add.at(g, m.ev[:, 12:], E[:, None] * Ku)
    np.add.at(g, m.fv[:, 4], -0.25 * mu.sum(axis=1) + x[m.nu0] / m.nelems)
    np.add.at(g, m.fv[:, 5:], rt @ m.A.T - 0.25 * re[:, None])
    fu = m.f[m.u0:m.u0 + 2 * m.nnodes]
    g[m.u0:m.u0 + 2 * m.nnodes] += alpha * fu
    g[m.lam0:m.lam0 + 2 * m.nnodes] -= fu
    g[m.nu0] += re.sum() / m.nelems - m.volfrac - x[m.s0]
    g[m.s0] += -x[m.nu0]
    return g


def hessian_dense_blocks(m, x):
    """Per-element 20x20 elasticity and 9x9 filter blocks."""
    u = x[m.ev[:, :8]]
    rt = x[m.ev[:, 8:12]]
    lam = x[m.ev[:, 12:]]
    E, dE, d2E = _stiffness(m, rt.mean(axis=1))
    Ku = u @ m.K0.T
    Kl = lam @ m.K0.T
    lKu = np.sum(lam * Ku, axis=1)
    ne = m.nelems
    H = np.zeros((ne, 20, 20))
    H[:, :8, 8:12] = 0.25 * (dE[:, None] * Kl)[:, :, None]
    H[:, 8:12, :8] = np.transpose(H[:, :8, 8:12], (0, 2, 1))
    H[:, :8, 12:] = E[:, None, None] * m.K0[None]
    H[:, 12:, :8] = E[:, None, None] * m.K0.T[None]
    H[:, 8:12, 8:12] = (0.0625 * d2E * lKu)[:, None, None]
    H[:, 12:, 8:12] = 0.25 * (dE[:, None] * Ku)[:, :, None]
    H[:, 8:12, 12:] = np.transpose(H[:, 12:, 8:12], (0, 2, 1))
    Fb = np.zeros((9, 9))
    Fb[5:, :4] = m.A
    Fb[:4, 5:] = m.A.T
    Fb[5:, 4] = -0.25
    Fb[4, 5:] = -0.25
    return H, Fb


def hessian_values(m, x, alpha=1.0):
    """KKT values on m's CSR pattern, fixed rows/columns applied."""
    vals = np.zeros(m.nnz)
    H, Fb = hessian_dense_blocks(m, x)
    np.add.at(vals, m.epos.ravel(), H.reshape(-1))
    np.add.at(vals, m.fpos.ravel(), np.broadcast_to(Fb.ravel(), (m.nelems, 81)).ravel())
    np.add.at(vals, m.vpos.ravel(), 1.0 / m.nelems)
    np.add.at(vals, m.spos, -1.0)
    vals[m.fixed_zero_pos] = 0.0
    vals[m.fixed_diag_pos] = 1.0
    return vals


def gradient_fixed(m, x, alpha=1.0):
    g = gradient(m, x, alpha)
    g[m.fixed] = 0.0
    return g
