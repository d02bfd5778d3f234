"""The interior-point driver (amigo_b200.optimizer.Optimizer) over the GPU
numeric core -- InteriorPointOptimizer, B200Solver and the device cart-pole
problem -- against the reference Optimizer's records on the host core
(tests/golden/ref_optimizer_cartpole.json, made by the reference's own
driver over its C++ backend and SparseLDL).  The GPU factor is a different
rounding of the same pivot sequence and iterative refinement brings each
direction to the same 1e-10 residual, so the runs agree to within one
iteration, the final objective to 1e-8 relative and the early records'
KKT error components to 1e-6 relative."""
import json
import os

import numpy as np
import pytest
import torch

from amigo_b200.ipm import InteriorPointOptimizer
from amigo_b200.ipm_driver import CartPoleProblem
from amigo_b200.optimizer import Optimizer
from amigo_b200.problems.cartpole import CartPole, batch_config
from amigo_b200.solver import B200Solver

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_optimizer_cartpole.json")


def run_gpu(m, dev="cuda:0"):
    P = CartPoleProblem(m, dev)
    S = B200Solver(P)
    x = torch.from_numpy(np.array(m.x0, dtype=np.float64)).to(dev)
    opt = Optimizer(P, x, np.asarray(m.lower, np.float64), np.asarray(m.upper, np.float64),
                    S, backend_class=InteriorPointOptimizer, device=dev)
    r = opt.optimize()
    xf = opt.vars.get_solution()
    return r, P.objective(xf), float(torch.linalg.norm(xf).item())


def _cases():
    B = batch_config(k=512, seed=0)
    return [("cartpole_N100_seed0", CartPole(N=100, seed=0))] + \
        [("batch512_seed0_inst%d" % i, B.inst[i]) for i in range(6)]


@pytest.mark.parametrize("name,m", _cases(), ids=[c[0] for c in _cases()])
def test_gpu_core_follows_reference_driver(name, m):
    want = json.load(open(GOLD))[name]
    r, obj, xn = run_gpu(m)
    assert r["converged"] == want["converged"]
    assert abs((len(r["iterations"]) - 1) - want["iterations"]) <= 1
    assert obj == pytest.approx(want["objective"], rel=1e-8)
    assert xn == pytest.approx(want["x_norm"], rel=1e-6)
    for a, b in list(zip(r["iterations"], want["records"]))[:4]:
        for k in ("barrier_param", "alpha_x", "alpha_z", "inf_pr", "inf_du", "compl"):
            if b[k] is not None:
                assert a[k] == pytest.approx(b[k], rel=1e-6, abs=1e-12), (a["iteration"], k)
