"""Cart-pole swing-up by trapezoidal direct collocation (the N = 100 config).

Stated from the config: N intervals over a fixed T = 2.0 s (h = T / N),
states (x, theta, xdot, thetadot), control u, frictionless cart-pole with
cart mass M = 1.0, point-mass pole m = 0.3 at l = 0.5, g = 9.81, theta
measured from the hanging position; objective the trapezoidal integral of
u^2; boundary states (0, 0, 0, 0) -> (1, pi, 0, 0); bounds |u| <= 20,
|x| <= 2; initial guess the linear interpolation of the boundary states plus
N(0, 0.01) noise from the seed.  The explicit dynamics are the standard
ones for this system (M. Kelly, "An Introduction to Trajectory
Optimization", SIAM Review 2017, cart-pole appendix):
    xdd = (l m sin(t) td^2 + u + m g cos(t) sin(t)) / (M + m (1 - cos(t)^2))
    tdd = -(l m cos(t) sin(t) td^2 + u cos(t) + (M + m) g sin(t))
          / (l M + l m (1 - cos(t)^2))
Variables per node k = 0..N: (x, theta, xdot, thetadot, u) -> 5 (N + 1)
primal; multipliers: 4 per interval (defects) and 8 boundary conditions.
For N = 100: 505 primal + 408 multipliers = 913 KKT rows.

Each interval is one component instance (its 10 node variables and its 4
defect multipliers); the two boundary-condition components hold a node's
4 states and 4 multipliers.  Derivatives are evaluated on the device with
hyper-dual numbers (csrc/cartpole.cu); this module builds numbering,
bounds, the KKT pattern and the CSR positions of every instance block.
"""
import numpy as np
import scipy.sparse as sp

M_CART, M_POLE, L_POLE, GRAV = 1.0, 0.3, 0.5, 9.81


class CartPole:
    def __init__(self, N=100, T=2.0, m_pole=M_POLE, xf=1.0, seed=0,
                 umax=20.0, xmax=2.0):
        self.N, self.T, self.h = N, T, T / N
        self.m_pole, self.xf = m_pole, xf
        nn = N + 1
        self.npr = 5 * nn
        self.d0 = self.npr                    # defect multipliers
        self.b0 = self.d0 + 4 * N             # boundary multipliers (8)
        self.n = self.b0 + 8
        self.mult = np.zeros(self.n, bool)
        self.mult[self.d0:] = True
        self.lower = np.full(self.n, -np.inf)
        self.upper = np.full(self.n, np.inf)
        var = lambda k, j: 5 * k + j
        for k in range(nn):
            self.lower[var(k, 0)], self.upper[var(k, 0)] = -xmax, xmax
            self.lower[var(k, 4)], self.upper[var(k, 4)] = -umax, umax
        self.lower[self.d0:] = 0.0           # constraint targets lbh
        q0 = np.zeros(4)
        qf = np.array([xf, np.pi, 0.0, 0.0])
        self.lower[self.b0:self.b0 + 4] = q0
        self.lower[self.b0 + 4:self.b0 + 8] = qf
        # interval instance: [q_k (4), u_k, q_k+1 (4), u_k+1 | lam (4)]
        k = np.arange(N)
        self.iv = np.stack([5 * k + j for j in range(5)] +
                           [5 * (k + 1) + j for j in range(5)] +
                           [self.d0 + 4 * k + j for j in range(4)],
                           axis=1).astype(np.int32)
        # boundary instances: [q (4) | mu (4)]
        self.bv = np.array([[0, 1, 2, 3] + [self.b0 + j for j in range(4)],
                            [5 * N + j for j in range(4)] +
                            [self.b0 + 4 + j for j in range(4)]], np.int32)
        self._pattern()
        r = np.random.RandomState(seed)
        t = np.linspace(0.0, 1.0, nn)
        x = np.zeros(self.n)
        for j in range(4):
            x[5 * np.arange(nn) + j] = q0[j] + (qf[j] - q0[j]) * t
        x[:self.npr] += r.normal(0.0, 0.01, self.npr)
        self.x0 = x

    def _pattern(self):
        n = self.n
        rows, cols = [], []
        for blk in (self.iv, self.bv):
            k = blk.shape[1]
            rows.append(np.repeat(blk, k, axis=1).ravel())
            cols.append(np.tile(blk, (1, k)).ravel())
        rows.append(np.arange(n))
        cols.append(np.arange(n))
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

        k = self.iv.shape[1]
        self.ipos = pos(np.repeat(self.iv, k, axis=1), np.tile(self.iv, (1, k))
                        ).reshape(len(self.iv), k * k)
        k = self.bv.shape[1]
        self.bpos = pos(np.repeat(self.bv, k, axis=1), np.tile(self.bv, (1, k))
                        ).reshape(2, k * k)
        self.diag_pos = pos(np.arange(n), np.arange(n))

    def device_model(self, device):
        from amigo_b200.fem import CartPoleDevice
        return CartPoleDevice(self, device)


class CartPoleBatch:
    """Independent cart-pole instances stored one after another (the
    batched-trajectories config: N ~ U{50..400}, pole mass ~ U(0.1, 0.5),
    final cart position ~ U(-1, 1), from the seed)."""

    def __init__(self, instances):
        self.inst = list(instances)
        self.k = len(self.inst)
        ns = [m.n for m in self.inst]
        self.var_off = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
        self.nnz_off = np.concatenate([[0], np.cumsum([m.nnz for m in self.inst])])
        self.n = int(self.var_off[-1])
        self.nnz = int(self.nnz_off[-1])
        cat = lambda f: np.concatenate([f(m) for m in self.inst])
        self.mult = cat(lambda m: m.mult)
        self.lower = cat(lambda m: m.lower)
        self.upper = cat(lambda m: m.upper)
        self.x0 = cat(lambda m: m.x0)
        voff = self.var_off.astype(np.int32)
        zoff = self.nnz_off.astype(np.int32)

        def shifted(name, offs, rows_of=None):
            # concatenation of each instance's int32 index array + its offset
            parts = [getattr(m, name) for m in self.inst]
            shape = (sum(a.shape[0] for a in parts),) + parts[0].shape[1:]
            out = np.empty(shape, np.int32)
            r = 0
            for a, o in zip(parts, offs):
                np.add(a, o, out=out[r:r + a.shape[0]], casting="unsafe")
                r += a.shape[0]
            return out

        self.iv = shifted("iv", voff)
        self.ipos = shifted("ipos", zoff)
        self.bv = shifted("bv", voff)
        self.bpos = shifted("bpos", zoff)
        self.h_iv = cat(lambda m: np.full(m.N, m.h))
        self.m_iv = cat(lambda m: np.full(m.N, m.m_pole))
        self.inst_iv = np.concatenate([[0], np.cumsum([m.N for m in self.inst])]).astype(np.int32)
        self.vinst = np.repeat(np.arange(self.k, dtype=np.int32), ns)
        self.diag_pos = shifted("diag_pos", zoff)
        self.N = int(self.inst_iv[-1])
        self.npr = int((~self.mult).sum())
        # block-diagonal CSR of the whole batch
        self.rowp = np.empty(self.n + 1, np.int32)
        self.rowp[0] = 0
        for m, a, o in zip(self.inst, self.var_off, zoff):
            np.add(m.rowp[1:], o, out=self.rowp[a + 1:a + 1 + m.n], casting="unsafe")
        self.cols = shifted("cols", voff)

    def patterns(self):
        return [(m.n, m.rowp, m.cols) for m in self.inst]

    def device_model(self, device):
        from amigo_b200.fem import CartPoleDevice
        return CartPoleDevice(self, device, batch=True)


def batch_config(k=512, seed=0, nmin=50, nmax=400):
    """The batched-trajectories config: k instances from the seed."""
    r = np.random.RandomState(seed)
    Ns = r.randint(nmin, nmax + 1, size=k)
    ms = r.uniform(0.1, 0.5, size=k)
    xfs = r.uniform(-1.0, 1.0, size=k)
    return CartPoleBatch([CartPole(N=int(N), m_pole=float(mp), xf=float(xf),
                                   seed=seed + 1 + i)
                          for i, (N, mp, xf) in enumerate(zip(Ns, ms, xfs))])
