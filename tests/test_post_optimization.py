"""Post-optimality sensitivities (amigo_b200.post_optimization, CPU part):
the generated cart-pole model optimised by amigo_b200.optimizer.Optimizer
over the host numeric core (the reference's C++ backend and SparseLDL,
oracle/_ref); d output / d data by the adjoint and the direct method agree
with each other to 1e-8 and with central finite differences of re-solved
optima to 1e-5.  Needs the reference sources (skipped otherwise)."""
import os

import numpy as np
import pytest

from amigo_b200.optimizer import Optimizer
from amigo_b200.post_optimization import PostOptimization
from amigo_b200.problems import components as C
from amigo_b200.problems.cartpole import CartPole

REF = os.environ.get("AMIGO_REF_ROOT", "/root/reference")
needs_ref = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "amigo", "algorithm")),
                               reason="reference sources absent")


def optimize(G, m):
    from oracle import ref_optimizer as RO
    alg = RO.install()
    P = RO.HostProblem(G, lambda x, a: G.host_derivatives(x, a)[0],
                       lambda x, a: G.host_derivatives(x, a)[1],
                       lambda x, a: G.host_lagrangian(x, a))
    solver = alg.solvers.AmigoSolver(P)
    x = RO.HostVector(arr=np.array(m.x0, dtype=np.float64))
    lo = RO.HostVector(arr=np.array(m.lower, dtype=np.float64))
    hi = RO.HostVector(arr=np.array(m.upper, dtype=np.float64))
    opt = Optimizer(P, x, lo, hi, solver, backend_class=RO.InteriorPointOptimizer)
    r = opt.optimize(dict(convergence_tolerance=1e-10))
    assert r["converged"]
    return opt


@needs_ref
def test_adjoint_direct_and_finite_differences(oracle_ref):
    m = CartPole(N=16, seed=1)
    G = C.cartpole_model(m)
    opt = optimize(G, m)
    post = PostOptimization(opt, G)
    out0 = post.compute_output()
    assert out0.shape == (2 * m.N,)
    # outputs: effort of interval 3, cart position at the end of intervals 9
    # and 15; data: the pole mass of intervals 2 and 11
    of, wrt = [3 * 2 + 0, 9 * 2 + 1, 15 * 2 + 1], [2 * 2 + 1, 11 * 2 + 1]
    A = post.compute_post_opt_derivatives(of, wrt, "adjoint")
    D = post.compute_post_opt_derivatives(of, wrt, "direct")
    assert np.allclose(A, D, rtol=1e-8, atol=1e-10)
    eps = 1e-5
    data = G.groups[0].data
    for j, w in enumerate(wrt):
        e, c = divmod(w, 2)
        v0 = data[e, c]
        outs = []
        for s in (1.0, -1.0):
            data[e, c] = v0 + s * eps
            o = optimize(G, m)
            outs.append(PostOptimization(o, G).compute_output()[of])
        data[e, c] = v0
        fd = (outs[0] - outs[1]) / (2 * eps)
        assert np.allclose(A[:, j], fd, rtol=1e-5, atol=1e-7), (j, A[:, j], fd)
