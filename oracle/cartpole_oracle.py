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


# ---------------------------------------------------------------------------
# Exact derivatives with vectorised hyper-dual numbers (same method as the
# device kernels: Fike & Alonso 2011), for host-side IPM runs.
class _HD:
    __slots__ = ("a", "b", "c", "d")
    __array_ufunc__ = None  # numpy arrays defer to the reflected operators

    def __init__(self, a, b=0.0, c=0.0, d=0.0):
        self.a, self.b, self.c, self.d = a, b, c, d

    @staticmethod
    def _w(y):
        return y if isinstance(y, _HD) else _HD(y)

    def __add__(self, y):
        y = self._w(y)
        return _HD(self.a + y.a, self.b + y.b, self.c + y.c, self.d + y.d)

    __radd__ = __add__

    def __sub__(self, y):
        y = self._w(y)
        return _HD(self.a - y.a, self.b - y.b, self.c - y.c, self.d - y.d)

    def __rsub__(self, y):
        return self._w(y) - self

    def __neg__(self):
        return _HD(-self.a, -self.b, -self.c, -self.d)

    def __mul__(self, y):
        y = self._w(y)
        return _HD(self.a * y.a, self.a * y.b + self.b * y.a,
                   self.a * y.c + self.c * y.a,
                   self.a * y.d + self.b * y.c + self.c * y.b + self.d * y.a)

    __rmul__ = __mul__

    def inv(self):
        r = 1.0 / self.a
        r2 = r * r
        return _HD(r, -r2 * self.b, -r2 * self.c, -r2 * self.d + 2.0 * r2 * r * self.b * self.c)

    def __truediv__(self, y):
        return self * self._w(y).inv()

    def __rtruediv__(self, y):
        return self._w(y) * self.inv()


def _sin(x):
    s, c = np.sin(x.a), np.cos(x.a)
    return _HD(s, c * x.b, c * x.c, c * x.d - s * x.b * x.c)


def _cos(x):
    s, c = np.sin(x.a), np.cos(x.a)
    return _HD(c, -s * x.b, -s * x.c, -s * x.d - c * x.b * x.c)


def _dyn_hd(q, u, m_pole):
    s, c = _sin(q[1]), _cos(q[1])
    td2 = q[3] * q[3]
    den = M_CART + m_pole * (1.0 - c * c)
    xdd = (L_POLE * m_pole * s * td2 + u + m_pole * GRAV * c * s) / den
    tdd = -(L_POLE * m_pole * c * s * td2 + u * c +
            (M_CART + m_pole) * GRAV * s) / (L_POLE * den)
    return [q[2], q[3], xdd, tdd]


def _node_derivs(m, z, lam, alpha):
    """phi(z) = alpha h/2 u^2 - h/2 lam^T f(z) over all nodes at once
    (z: [K, 5], lam: [K, 4]): gradient [K, 5], Hessian [K, 5, 5], Jacobian
    of f [K, 4, 5]."""
    K = z.shape[0]
    hh = 0.5 * m.h
    grad = np.zeros((K, 5))
    hess = np.zeros((K, 5, 5))
    jac = np.zeros((K, 4, 5))
    for i in range(5):
        for j in range(i, 5):
            zz = [_HD(z[:, t].copy(), np.zeros(K), np.zeros(K), np.zeros(K)) for t in range(5)]
            zz[i].b = np.ones(K)
            zz[j].c = zz[j].c + 1.0
            f = _dyn_hd(zz[:4], zz[4], m.m_pole)
            phi = alpha * hh * zz[4] * zz[4]
            for t in range(4):
                phi = phi - hh * lam[:, t] * f[t]
            hess[:, i, j] = phi.d
            hess[:, j, i] = phi.d
            if i == j:
                grad[:, i] = phi.b
                for t in range(4):
                    jac[:, t, i] = f[t].b
    return grad, hess, jac


def gradient(m, x, alpha=1.0):
    """nabla L (primal rows) and constraint values (multiplier rows)."""
    g = np.zeros(m.n)
    z0 = x[m.iv[:, 0:5]]
    z1 = x[m.iv[:, 5:10]]
    lam = x[m.iv[:, 10:14]]
    g0, _, _ = _node_derivs(m, z0, lam, alpha)
    g1, _, _ = _node_derivs(m, z1, lam, alpha)
    g0[:, :4] -= lam
    g1[:, :4] += lam
    np.add.at(g, m.iv[:, 0:5], g0)
    np.add.at(g, m.iv[:, 5:10], g1)
    g[m.d0:] += constraints(m, x)[m.d0:]
    g[0:4] += x[m.b0:m.b0 + 4]
    g[5 * m.N:5 * m.N + 4] += x[m.b0 + 4:m.b0 + 8]
    return g


def hessian_values(m, x, alpha=1.0):
    vals = np.zeros(m.nnz)
    z0 = x[m.iv[:, 0:5]]
    z1 = x[m.iv[:, 5:10]]
    lam = x[m.iv[:, 10:14]]
    _, h0, j0 = _node_derivs(m, z0, lam, alpha)
    _, h1, j1 = _node_derivs(m, z1, lam, alpha)
    K = m.N
    blk = np.zeros((K, 14, 14))
    blk[:, 0:5, 0:5] = h0
    blk[:, 5:10, 5:10] = h1
    eye = np.zeros((4, 5))
    eye[np.arange(4), np.arange(4)] = 1.0
    A = -eye[None] - 0.5 * m.h * j0
    B = eye[None] - 0.5 * m.h * j1
    blk[:, 10:14, 0:5] = A
    blk[:, 0:5, 10:14] = np.transpose(A, (0, 2, 1))
    blk[:, 10:14, 5:10] = B
    blk[:, 5:10, 10:14] = np.transpose(B, (0, 2, 1))
    np.add.at(vals, m.ipos.ravel(), blk.reshape(-1))
    for b in range(2):
        for t in range(4):
            vals[m.bpos[b, (4 + t) * 8 + t]] += 1.0
            vals[m.bpos[b, t * 8 + 4 + t]] += 1.0
    return vals
