"""CPU restatement of the cart-pole collocation Lagrangian (test
infrastructure only; numpy).  The reference's cart-pole example uses an
implicit formulation with extra variables (examples/trajectory/cart/
cart_pole.py:49-91); this config is the explicit one, so its derivatives are
pinned by finite differences of this Lagrangian ("parity unpinned" against
the reference itself)."""
import numpy as np

from amigo_b200.problems.cartpole import GRAV, L_POLE, M_CART


def dynamics(q, u, m_pole):
    x, t, xd, td = q
    s, c = np.sin(t), np.cos(t)
    den = M_CART + m_pole * (1.0 - c * c)
    xdd = (L_POLE * m_pole * s * td * td + u + m_pole * GRAV * c * s) / den
    tdd = -(L_POLE * m_pole * c * s * td * td + u * c +
            (M_CART + m_pole) * GRAV * s) / (L_POLE * den)
    return np.array([xd, td, xdd, tdd])


def constraints(m, x):
    """Constraint values at the multiplier rows (defects, boundary states)."""
    c = np.zeros(m.n)
    for k in range(m.N):
        z0 = x[5 * k:5 * k + 5]
        z1 = x[5 * (k + 1):5 * (k + 1) + 5]
        d = z1[:4] - z0[:4] - 0.5 * m.h * (dynamics(z0[:4], z0[4], m.m_pole) +
                                           dynamics(z1[:4], z1[4], m.m_pole))
        c[m.d0 + 4 * k:m.d0 + 4 * k + 4] = d
    c[m.b0:m.b0 + 4] = x[0:4]
    c[m.b0 + 4:m.b0 + 8] = x[5 * m.N:5 * m.N + 4]
    return c


def objective(m, x):
    u = x[4:m.npr:5]
    return float(np.sum(0.5 * m.h * (u[:-1] ** 2 + u[1:] ** 2)))


def lagrangian(m, x, alpha=1.0):
    return alpha * objective(m, x) + float(x[m.d0:] @ constraints(m, x)[m.d0:])
