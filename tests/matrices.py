"""Test matrices.

`ldl_unit_matrix` and `poisson_2d` restate the known-answer matrices of the
reference's tests/unit/test_ldl.py:20-118 (seven small symmetric matrices,
including cases that need 2x2 pivots, and the randomly permuted 5-point
Laplacian with np.random.seed(0)).  `kkt_matrix` builds seeded saddle-point
matrices shaped like amigo's KKT systems: an SPD-plus-indefinite Hessian block
and a constraint Jacobian with a zero or -delta_c multiplier block.
"""
import numpy as np
import scipy.sparse as sp

UNIT_MATRICES = [
    [[2, 1, 0, 0, 0], [1, 2, 1, 0, 0], [0, 1, 2, 1, 0], [0, 0, 1, 2, 1],
     [0, 0, 0, 1, 2]],
    [[0, 1, 0, 0, 0], [1, 0, 1, 0, 0], [0, 1, 2, 1, 0], [0, 0, 1, 2, 1],
     [0, 0, 0, 1, 2]],
    [[0, 0, 0, 1, 1], [0, 0, 1, 0, 1], [0, 1, 2, 0, 1], [1, 0, 0, 0, 1],
     [1, 1, 1, 1, 0]],
    [[0, 1, 0, 0, 1], [1, 0, 2, 0, 1], [0, 2, 0, 0, 1], [0, 0, 0, 2, 1],
     [1, 1, 1, 1, 0]],
    [[0, 1], [1, 0]],
    [[1, 1], [1, 0]],
    [[1, 2, 3], [2, 1, 3], [3, 3, 0]],
]
# Inertia stated by the reference test for matrices 0 and 1; the others are
# computed from eigenvalues there as here.
UNIT_INERTIA = {0: (5, 0), 1: (4, 1)}


def eig_inertia(A, tol=1e-12):
    w = np.linalg.eigvalsh(np.asarray(A, dtype=float))
    assert np.min(np.abs(w)) >= tol
    return int(np.sum(w >= 0)), int(np.sum(w < 0))


def ldl_unit_matrix(index):
    A = np.array(UNIT_MATRICES[index], dtype=float)
    inertia = UNIT_INERTIA.get(index, eig_inertia(A))
    M = sp.csr_matrix(A)  # explicit zeros (e.g. zero diagonals) are dropped
    return M, inertia


def poisson_2d(n, seed=0):
    m = n - 1
    h = 1.0 / n
    T = sp.diags([-np.ones(m - 1), 2.0 * np.ones(m), -np.ones(m - 1)],
                 [-1, 0, 1], format="csr")
    I = sp.eye(m, format="csr")
    A = ((sp.kron(I, T) + sp.kron(T, I)) / h**2).tocsr()
    perm = np.random.RandomState(seed).permutation(m * m)
    A = A[perm, :][:, perm].tocsr()
    return A, (m * m, 0)


def kkt_matrix(n_primal, n_con, seed, density=None, delta_c=0.0,
               indefinite=0.3, sort=True):
    """Random saddle-point matrix [[H, J^T], [J, -delta_c I]] with the
    multiplier rows interleaved among the primal rows (as amigo numbers
    them after its model-level reordering)."""
    r = np.random.RandomState(seed)
    if density is None:
        density = min(1.0, 6.0 / max(n_primal, 1))
    B = sp.random(n_primal, n_primal, density=density, random_state=r)
    H = (B + B.T).tocsr()
    d = np.abs(H).sum(axis=1).A1 + 1.0
    sign = np.where(r.rand(n_primal) < indefinite, -0.05, 1.0)
    H = H + sp.diags(d * sign)
    J = sp.random(n_con, n_primal, density=min(1.0, 4.0 / max(n_primal, 1)),
                  random_state=r).tolil()
    # full row rank: one strong entry per row, in distinct columns
    strong = np.resize(r.permutation(n_primal), n_con)
    for i in range(n_con):
        J[i, strong[i]] = 2.0 + r.rand()
    J = J.tocsr()
    C = -delta_c * sp.eye(n_con) if delta_c else sp.csr_matrix((n_con, n_con))
    K = sp.bmat([[H, J.T], [J, C]]).tocsr()
    n = n_primal + n_con
    p = r.permutation(n)
    K = K[p, :][:, p].tocsr()
    # keep a structural diagonal everywhere (amigo's KKT pattern has one)
    K = K.tocoo()
    rows = np.concatenate([K.row, np.arange(n)])
    cols = np.concatenate([K.col, np.arange(n)])
    vals = np.concatenate([K.data, np.zeros(n)])
    K = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    K.sum_duplicates()
    if sort:
        K.sort_indices()
    return K


def csr_arrays(M):
    M = M.tocsr()
    return (M.shape[0], np.ascontiguousarray(M.indptr, dtype=np.int32),
            np.ascontiguousarray(M.indices, dtype=np.int32),
            np.ascontiguousarray(M.data, dtype=np.float64))
