"""3D SIMP compliance cantilever in full space (the 48 x 24 x 24 config).

Model (stated from the config: unit trilinear hexahedra, 2x2x2 Gauss,
E0 = 1, Emin = 1e-9, nu = 0.3, penalty p = 3, Helmholtz density filter of
radius 1.5 elements, the x = 0 face clamped, a unit total load spread
evenly over the nodes of the bottom edge (y = 0) of the x = L face,
pointing in -y, volume fraction <= 0.3; element densities start at
0.3 + U(-0.01, 0.01) from the seed).  The Lagrangian and the variable
blocks are those of the 2D model (problems/simp2d.py) with hexahedra in
place of quads: per element u (24), filtered nodal densities (8) and
equilibrium multipliers (24) in the elasticity block, and rt (8), re,
filter multipliers (8) in the filter block; K(rt) = sum_e E(mean(rt_e)) K0.

Sizes: 30,625 nodes -> 91,875 displacements, 27,648 element densities,
30,625 filtered nodal densities, the volume slack, and 91,875 + 30,625 + 1
multipliers: n = 272,650 KKT rows.
"""
import numpy as np
import scipy.sparse as sp

from .simp2d import E0, EMIN, NU, PENALTY

GAUSS = (-1.0 / np.sqrt(3.0), 1.0 / np.sqrt(3.0))
# corner signs of the 8-node hexahedron (x fastest, then y, then z)
HEX = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)


def hex_shape(xi, eta, zeta):
    a, b, c = HEX[:, 0], HEX[:, 1], HEX[:, 2]
    N = 0.125 * (1 + a * xi) * (1 + b * eta) * (1 + c * zeta)
    Nxi = 0.125 * a * (1 + b * eta) * (1 + c * zeta)
    Neta = 0.125 * b * (1 + a * xi) * (1 + c * zeta)
    Nzeta = 0.125 * c * (1 + a * xi) * (1 + b * eta)
    return N, Nxi, Neta, Nzeta


def element_matrices(h=1.0, nu=NU):
    """Unit-modulus isotropic stiffness K0 (24x24, dofs ordered
    [u0 v0 w0 u1 ...]), consistent mass M (8x8) and Laplacian KL (8x8) of an
    h^3 trilinear cube, 2x2x2 Gauss."""
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    G = 1.0 / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[0, 0] = D[1, 1] = D[2, 2] = lam + 2 * G
    D[3, 3] = D[4, 4] = D[5, 5] = G
    K0 = np.zeros((24, 24))
    M = np.zeros((8, 8))
    KL = np.zeros((8, 8))
    detJ = (0.5 * h) ** 3
    for zeta in GAUSS:
        for eta in GAUSS:
            for xi in GAUSS:
                N, Nxi, Neta, Nzeta = hex_shape(xi, eta, zeta)
                Nx, Ny, Nz = Nxi * 2.0 / h, Neta * 2.0 / h, Nzeta * 2.0 / h
                B = np.zeros((6, 24))
                B[0, 0::3] = Nx
                B[1, 1::3] = Ny
                B[2, 2::3] = Nz
                B[3, 0::3] = Ny
                B[3, 1::3] = Nx
                B[4, 1::3] = Nz
                B[4, 2::3] = Ny
                B[5, 0::3] = Nz
                B[5, 2::3] = Nx
                K0 += B.T @ D @ B * detJ
                M += np.outer(N, N) * detJ
                KL += (np.outer(Nx, Nx) + np.outer(Ny, Ny) + np.outer(Nz, Nz)) * detJ
    return K0, M, KL


def csr_pattern(n, blocks, extra_pairs):
    """Sorted CSR pattern with the diagonal: all pairs inside each block row
    of every (nelem x k) block table, plus explicit (row, col) pairs.
    Built node-row by node-row in chunks to bound host memory."""
    rows, cols = [], []
    for blk in blocks:
        k = blk.shape[1]
        for s in range(0, len(blk), 4096):
            b = blk[s:s + 4096]
            rows.append(np.repeat(b, k, axis=1).ravel())
            cols.append(np.tile(b, (1, k)).ravel())
    for r, c in extra_pairs:
        rows.append(np.asarray(r).ravel())
        cols.append(np.asarray(c).ravel())
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    key = np.unique(np.concatenate(rows).astype(np.int64) * n +
                    np.concatenate(cols).astype(np.int64))
    r = (key // n).astype(np.int64)
    rowp = np.zeros(n + 1, np.int64)
    np.add.at(rowp, r + 1, 1)
    return np.cumsum(rowp).astype(np.int32), (key % n).astype(np.int32), key


class Simp3D:
    """Mesh, numbering, bounds, KKT pattern and element index maps; the
    attribute names follow problems.simp2d.Simp2D."""

    dim = 3
    nv = 8

    def __init__(self, nx=48, ny=24, nz=24, volfrac=0.3, rfilter=1.5, seed=0):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.volfrac = volfrac
        self.rfilter = rfilter
        nn = (nx + 1) * (ny + 1) * (nz + 1)
        ne = nx * ny * nz
        self.nnodes, self.nelems = nn, ne
        node = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)
        kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx),
                                 indexing="ij")
        ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
        self.conn = np.stack([node(ii + a, jj + b, kk + c) for a, b, c in
                              ((HEX + 1) // 2).astype(int)], axis=1)
        self.color = (ii % 2) + 2 * (jj % 2) + 4 * (kk % 2)

        o = 0
        self.u0 = o; o += 3 * nn
        self.rt0 = o; o += nn
        self.re0 = o; o += ne
        self.s0 = o; o += 1
        self.lam0 = o; o += 3 * nn
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
        self.upper[self.s0] = 0.0
        self.lower[self.lam0:] = 0.0

        # unit total load in -y spread over the bottom edge of the x = L face
        edge = node(nx, 0, np.arange(nz + 1))
        self.f = np.zeros(self.n)
        self.f[self.u0 + 3 * edge + 1] = -1.0 / len(edge)
        # clamped x = 0 face: displacements and their multipliers fixed
        J, K = np.meshgrid(np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
        face = node(0, J.ravel(), K.ravel())
        fixed = np.concatenate([self.u0 + 3 * face + d for d in range(3)] +
                               [self.lam0 + 3 * face + d for d in range(3)])
        self.fixed = np.sort(fixed).astype(np.int32)
        # a fixed row is an identity row, not a constraint: the fixed
        # multipliers leave the multiplier set (they are neither bounded
        # nor counted among the constraints an inertia check expects)
        self.mult[self.fixed] = False
        self.lower[self.fixed] = -np.inf
        self.upper[self.fixed] = np.inf

        c = self.conn
        udofs = np.stack([3 * c[:, a] + d for a in range(8) for d in range(3)], axis=1)
        self.ev = np.concatenate([self.u0 + udofs, self.rt0 + c, self.lam0 + udofs],
                                 axis=1).astype(np.int32)
        self.fv = np.concatenate([self.rt0 + c, (self.re0 + np.arange(ne))[:, None],
                                  self.mu0 + c], axis=1).astype(np.int32)
        self.K0, self.M, self.KL = element_matrices()
        self.rlen = rfilter / (2.0 * np.sqrt(3.0))
        self.A = self.M + self.rlen ** 2 * self.KL
        self.Bq = 1.0 / 8.0
        self._pattern()
        r = np.random.RandomState(seed)
        self.re_init = volfrac + r.uniform(-0.01, 0.01, ne)

    def _pattern(self):
        n, ne = self.n, self.nelems
        re = self.re0 + np.arange(ne)
        nuv = np.full(ne, self.nu0)
        extra = [(re, nuv), (nuv, re), ([self.s0, self.nu0], [self.nu0, self.s0])]
        self.rowp, self.cols, keys = csr_pattern(n, (self.ev, self.fv), extra)
        self.nnz = int(self.rowp[-1])

        def pos(rr, cc):
            q = np.asarray(rr, np.int64) * n + np.asarray(cc, np.int64)
            p = np.searchsorted(keys, q)
            assert np.all(keys[p] == q)
            return p.astype(np.int32)

        k = self.ev.shape[1]
        self.epos = np.empty((ne, k * k), np.int32)
        for s in range(0, ne, 4096):
            b = self.ev[s:s + 4096]
            self.epos[s:s + 4096] = pos(np.repeat(b, k, axis=1),
                                        np.tile(b, (1, k))).reshape(len(b), k * k)
        k = self.fv.shape[1]
        self.fpos = pos(np.repeat(self.fv, k, axis=1), np.tile(self.fv, (1, k))
                        ).reshape(ne, k * k)
        self.vpos = np.stack([pos(re, nuv), pos(nuv, re)], 1).astype(np.int32)
        self.spos = np.array([pos([self.s0], [self.nu0])[0],
                              pos([self.nu0], [self.s0])[0]], np.int32)
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
        x = np.zeros(self.n)
        cnt = np.zeros(self.nnodes)
        acc = np.zeros(self.nnodes)
        np.add.at(acc, self.conn.ravel(), np.repeat(self.re_init, 8))
        np.add.at(cnt, self.conn.ravel(), 1.0)
        x[self.rt0:self.rt0 + self.nnodes] = acc / cnt
        x[self.re0:self.re0 + self.nelems] = self.re_init
        x[self.s0] = min(self.re_init.mean() - self.volfrac, -1e-3)
        return x

    def color_lists(self):
        return [np.nonzero(self.color == c)[0].astype(np.int32) for c in range(8)]

    def device_model(self, device):
        from amigo_b200.fem import Simp3DDevice
        return Simp3DDevice(self, device)
