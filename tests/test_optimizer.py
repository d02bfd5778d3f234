"""The interior-point driver (amigo_b200.optimizer.Optimizer) against the
reference's own driver (CPU only; needs the reference sources).

Both drivers run over the same host numeric core -- the reference's
interior_point_backend.h functions and SparseLDL (oracle/_ref) behind the
reference's backend interface, with the reference's own AmigoSolver and its
iterative refinement -- so every decision (barrier updates, inertia
corrections, line-search trials, step lengths) and every iterate must
agree, and every record equals the golden one bit for bit.  The golden records come from tests/golden/make_ref_optimizer_golden.py
(the reference Optimizer on the cart-pole configuration and six batched
instances)."""
import json
import os

import numpy as np
import pytest

from amigo_b200.optimizer import Optimizer
from amigo_b200.problems.cartpole import CartPole, batch_config

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_optimizer_cartpole.json")
REF = os.environ.get("AMIGO_REF_ROOT", "/root/reference")
needs_ref = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "amigo", "algorithm")),
                               reason="reference sources absent")
FIELDS = ("residual", "barrier_param", "alpha_x", "alpha_z", "line_iters",
          "inertia_delta", "inf_pr", "inf_du", "compl", "nlp_error", "objective")


def _host_run(m, oracle_ref):
    from oracle import cartpole_oracle as CO
    from oracle import ref_optimizer as RO
    alg = RO.install()
    P = RO.HostProblem(m, lambda x, a: CO.gradient(m, x, a),
                       lambda x, a: CO.hessian_values(m, x, a),
                       lambda x, a: CO.lagrangian(m, x, a))
    solver = alg.solvers.AmigoSolver(P)
    x = RO.HostVector(arr=np.array(m.x0, dtype=np.float64))
    lo = RO.HostVector(arr=np.array(m.lower, dtype=np.float64))
    hi = RO.HostVector(arr=np.array(m.upper, dtype=np.float64))
    opt = Optimizer(P, x, lo, hi, solver, backend_class=RO.InteriorPointOptimizer)
    return opt.optimize()


def _cases():
    B = batch_config(k=512, seed=0)
    return [("cartpole_N100_seed0", CartPole(N=100, seed=0))] + \
        [("batch512_seed0_inst%d" % i, B.inst[i]) for i in range(6)]


@needs_ref
@pytest.mark.parametrize("name,m", _cases(), ids=[c[0] for c in _cases()])
def test_driver_reproduces_reference_iterations(oracle_ref, name, m):
    want = json.load(open(GOLD))[name]
    got = _host_run(m, oracle_ref)
    assert got["converged"] == want["converged"]
    recs = got["iterations"]
    assert len(recs) - 1 == want["iterations"]
    for a, b in zip(recs, want["records"]):
        for k in FIELDS:
            if b[k] is None:
                continue
            assert a[k] == b[k], (a["iteration"], k)
