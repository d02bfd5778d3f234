"""2D SIMP compliance in full space (the 128 x 64 plane-stress config).

Model (stated from the config: unit bilinear quads, E0 = 1, Emin = 1e-9,
nu = 0.3, penalty p = 3, left edge clamped, unit downward point load at the
mid-node of the right edge, volume fraction <= 0.4, Helmholtz density
filter of radius 1.5 elements; element densities start at
0.4 + U(-0.01, 0.01) from the seed).  The component split follows the
reference's compliance example (examples/compliance_helmholtz/
compliance.py:66-233): a per-element elasticity component with nodal
displacements, filtered nodal densities and equilibrium residuals, a
per-element Helmholtz filter component, and a volume component.

Variables (block numbering): u (2 per node), filtered nodal density rt,
element density re, the volume slack s; multipliers: equilibrium lam
(2 per node), filter mu (1 per node), volume nu.  The Lagrangian is
    L = f^T u + lam^T (K(rt) u - f) + mu^T (A rt - B re) + nu (v^T re - 0.4 - s)
with K(rt) = sum_e E(mean(rt_e)) K0_e, E(r) = Emin + r^p (E0 - Emin),
A = M + r_f^2 K_lap, B_ke = |e| / 4, v_e = 1 / nelem.  The clamped
displacements and their equilibrium multipliers are fixed variables: their
KKT rows/columns are zeroed with a unit diagonal, as the reference's
FixedVariables::zero_rows_and_columns does (include/fixed_variables.h:66-72).

Every numeric evaluation (gradient, Hessian scatter into the CSR KKT
pattern, fixed-row handling) runs in libamigo_b200.so's element kernels;
this module only builds the mesh, the numbering and the index maps.
"""
import numpy as np
import scipy.sparse as sp

E0, EMIN, NU, PENALTY = 1.0, 1e-9, 0.3, 3.0
GAUSS = (-1.0 / np.sqrt(3.0), 1.0 / np.sqrt(3.0))


def quad_shape(xi, eta):
    N = 0.25 * np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta),
                         (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)])
    Nxi = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
    Neta = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
    return N, Nxi, Neta


def element_matrices(h=1.0, nu=NU):
    """Unit-modulus plane-stress stiffness K0 (8x8, dofs ordered
    [u0 v0 u1 v1 u2 v2 u3 v3]), consistent mass M (4x4) and Laplacian
    KL (4x4) of an h x h bilinear square, 2x2 Gauss."""
    D = 1.0 / (1 - nu * nu) * np.array([[1, nu, 0], [nu, 1, 0],
                                        [0, 0, 0.5 * (1 - nu)]])
    K0 = np.zeros((8, 8))
    M = np.zeros((4, 4))
    KL = np.zeros((4, 4))
    detJ = 0.25 * h * h
    for eta in GAUSS:
        for xi in GAUSS:
            N, Nxi, Neta = quad_shape(xi, eta)
            Nx, Ny = Nxi * 2.0 / h, Neta * 2.0 / h
            Bm = np.zeros((3, 8))
            Bm[0, 0::2] = Nx
            Bm[1, 1::2] = Ny
            Bm[2, 0::2] = Ny
            Bm[2, 1::2] = Nx
            K0 += Bm.T @ D @ Bm * detJ
            M += np.outer(N, N) * detJ
            KL += (np.outer(Nx, Nx) + np.outer(Ny, Ny)) * detJ
    return K0, M, KL


class Simp2D:
    """Mesh, numbering, bounds, KKT pattern and element index maps."""

    def __init__(self, nx=128, ny=64, volfrac=0.4, rfilter=1.5, seed=0):
        self.nx, self.ny = nx, ny
        self.volfrac = volfrac
        self.rfilter = rfilter
        nn = (nx + 1) * (ny + 1)
        ne = nx * ny
        self.nnodes, self.nelems = nn, ne
        node = lambda i, j: i + j * (nx + 1)
        ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
        ii, jj = ii.ravel(), jj.ravel()
        self.conn = np.stack([node(ii, jj), node(ii + 1, jj),
                              node(ii + 1, jj + 1), node(ii, jj + 1)], axis=1)
        self.color = (ii % 2) + 2 * (jj % 2)  # no two same-colour elements share a node

        # numbering
        o = 0
        self.u0 = o; o += 2 * nn
        self.rt0 = o; o += nn
        self.re0 = o; o += ne
        self.s0 = o; o += 1
        self.lam0 = o; o += 2 * nn
        self.mu0 = o; o += nn
        self.nu0 = o; o += 1
        self.n = o
        self.mult = np.zeros(self.n, bool)
        self.mult[self.lam0:] = True

        self.lower = np.full(self.n, -np.inf)
        self.upper = np.full(self.n, np.inf)
        self.lower[self.rt0:self.rt0 + nn] = 0.0
        self.upper[self.rt0:self.rt0 + nn] = 1.0
        self.lower[self.re0:self.re0 + ne] = 0.0
        self.upper[self.re0:self.re0 + ne] = 1.0
        self.upper[self.s0] = 0.0            # v^T re - volfrac - s = 0, s <= 0
        self.lower[self.lam0:] = 0.0         # constraint targets lbh = 0

        # load: unit downward point load at the right mid-edge node
        self.f = np.zeros(self.n)
        self.load_node = node(nx, ny // 2)
        self.f[self.u0 + 2 * self.load_node + 1] = -1.0

        # clamped left edge: u, v and their equilibrium multipliers fixed
        left = node(0, np.arange(ny + 1))
        fixed = np.concatenate([self.u0 + 2 * left, self.u0 + 2 * left + 1,
                                self.lam0 + 2 * left, self.lam0 + 2 * left + 1])
        self.fixed = np.sort(fixed).astype(np.int32)
        # a fixed row is an identity row, not a constraint: the fixed
        # multipliers leave the multiplier set (they are neither bounded
        # nor counted among the constraints an inertia check expects)
        self.mult[self.fixed] = False
        self.lower[self.fixed] = -np.inf
        self.upper[self.fixed] = np.inf

        # element variable tables
        c = self.conn
        udofs = np.stack([2 * c[:, 0], 2 * c[:, 0] + 1, 2 * c[:, 1], 2 * c[:, 1] + 1,
                          2 * c[:, 2], 2 * c[:, 2] + 1, 2 * c[:, 3], 2 * c[:, 3] + 1],
                         axis=1)
        # elasticity block: [u (8) | rt (4) | lam (8)]
        self.ev = np.concatenate([self.u0 + udofs, self.rt0 + c, self.lam0 + udofs],
                                 axis=1).astype(np.int32)
        # filter block: [rt (4) | re (1) | mu (4)]
        self.fv = np.concatenate([self.rt0 + c, (self.re0 + np.arange(ne))[:, None],
                                  self.mu0 + c], axis=1).astype(np.int32)
        self.K0, self.M, self.KL = element_matrices()
        # Helmholtz length from the filter radius (r = R / (2 sqrt 3))
        self.rlen = rfilter / (2.0 * np.sqrt(3.0))
        self.A = self.M + self.rlen ** 2 * self.KL
        self._pattern()

        r = np.random.RandomState(seed)
        self.re_init = volfrac + r.uniform(-0.01, 0.01, ne)

    # -- KKT pattern (all pairs inside each component instance, plus the
    # diagonal), as OptimizationProblem::create_matrix builds it
    # (include/optimization_problem.h:596-682).
    def _pattern(self):
        n, ne = self.n, self.nelems
        rows, cols = [], []
        for blk in (self.ev, self.fv):
            k = blk.shape[1]
            rows.append(np.repeat(blk, k, axis=1).ravel())
            cols.append(np.tile(blk, (1, k)).ravel())
        vol = np.stack([self.re0 + np.arange(ne), np.full(ne, self.nu0)], 1)
        rows.append(np.repeat(vol, 2, axis=1).ravel())
        cols.append(np.tile(vol, (1, 2)).ravel())
        sl = np.array([[self.s0, self.nu0]])
        rows.append(np.repeat(sl, 2, axis=1).ravel())
        cols.append(np.tile(sl, (1, 2)).ravel())
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

        k = self.ev.shape[1]
        self.epos = pos(np.repeat(self.ev, k, axis=1), np.tile(self.ev, (1, k))
                        ).reshape(ne, k * k)
        k = self.fv.shape[1]
        self.fpos = pos(np.repeat(self.fv, k, axis=1), np.tile(self.fv, (1, k))
                        ).reshape(ne, k * k)
        re = self.re0 + np.arange(ne)
        self.vpos = np.stack([pos(re, np.full(ne, self.nu0)),
                              pos(np.full(ne, self.nu0), re)], 1).astype(np.int32)
        self.spos = np.array([pos(np.array([self.s0]), np.array([self.nu0]))[0],
                              pos(np.array([self.nu0]), np.array([self.s0]))[0]],
                             np.int32)
        self.diag_pos = pos(np.arange(n), np.arange(n))
        isf = np.zeros(n, bool)
        isf[self.fixed] = True
        rr = np.repeat(np.arange(n), np.diff(self.rowp))
        zero = (isf[rr] | isf[self.cols]) & (rr != self.cols)
        self.fixed_zero_pos = np.nonzero(zero)[0].astype(np.int32)
        self.fixed_diag_pos = self.diag_pos[self.fixed].astype(np.int32)

    @property
    def x0(self):
        """The initial point (initial_point()), as the IPM driver reads it."""
        return self.initial_point()

    def initial_point(self):
        """x0: u = 0, rt from the element densities averaged to nodes,
        re = 0.4 + U(-0.01, 0.01), s = v^T re - 0.4 clipped below 0,
        multipliers 0."""
        x = np.zeros(self.n)
        cnt = np.zeros(self.nnodes)
        acc = np.zeros(self.nnodes)
        np.add.at(acc, self.conn.ravel(), np.repeat(self.re_init, 4))
        np.add.at(cnt, self.conn.ravel(), 1.0)
        x[self.rt0:self.rt0 + self.nnodes] = acc / cnt
        x[self.re0:self.re0 + self.nelems] = self.re_init
        x[self.s0] = min(self.re_init.mean() - self.volfrac, -1e-3)
        return x

    def color_lists(self):
        return [np.nonzero(self.color == c)[0].astype(np.int32) for c in range(4)]

    def device_model(self, device):
        """Upload the index maps and constants; returns a Simp2DDevice."""
        from amigo_b200.fem import Simp2DDevice
        return Simp2DDevice(self, device)


def make(nx=128, ny=64, seed=0):
    return Simp2D(nx, ny, seed=seed)

