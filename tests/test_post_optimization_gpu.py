"""Post-optimality sensitivities on the GPU core: the generated cart-pole
model optimised by amigo_b200.optimizer.Optimizer over
InteriorPointOptimizer, B200Solver and the generated device kernels; the
adjoint and direct derivatives (each one multi-right-hand-side solve on the
resident factor) agree with each other to 1e-8 and with central finite
differences of re-solved optima to 1e-5."""
import numpy as np
import pytest
import torch

from amigo_b200.ipm import InteriorPointOptimizer
from amigo_b200.ipm_driver import GeneratedProblem
from amigo_b200.optimizer import Optimizer
from amigo_b200.post_optimization import PostOptimization
from amigo_b200.problems import components as C
from amigo_b200.problems.cartpole import CartPole
from amigo_b200.solver import B200Solver

pytestmark = pytest.mark.gpu


def optimize(G, m, dev="cuda:0"):
    P = GeneratedProblem(G, dev)
    S = B200Solver(P)
    x = torch.from_numpy(np.array(m.x0, dtype=np.float64)).to(dev)
    opt = Optimizer(P, x, np.asarray(m.lower, np.float64), np.asarray(m.upper, np.float64),
                    S, backend_class=InteriorPointOptimizer, device=dev)
    r = opt.optimize(dict(convergence_tolerance=1e-10))
    assert r["converged"]
    return opt


def test_adjoint_direct_and_finite_differences_on_device():
    m = CartPole(N=16, seed=1)
    G = C.cartpole_model(m)
    opt = optimize(G, m)
    post = PostOptimization(opt, G)
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
            outs.append(PostOptimization(optimize(G, m), G).compute_output()[of])
        data[e, c] = v0
        fd = (outs[0] - outs[1]) / (2 * eps)
        assert np.allclose(A[:, j], fd, rtol=1e-5, atol=1e-7), (j, A[:, j], fd)
