"""Generate tests/golden/ref_optimizer_cartpole.json: the reference's own
interior-point driver (amigo/algorithm/ipm_driver.py Optimizer, default
options, its AmigoSolver) run on the host over the reference's own C++
numeric core (oracle/ref_optimizer.py), on the cart-pole configuration
(N = 100, seed 0) and on the first instances of the 512-instance batched
configuration.  Per case: convergence, iteration count, final objective,
the final iterate's norm and the per-iteration records (residual, barrier
parameter, step lengths, line-search trials, inertia perturbation, the
scaled KKT error components and the barrier objective).

    python tests/golden/make_ref_optimizer_golden.py      # needs the reference sources
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from amigo_b200.problems.cartpole import CartPole, batch_config  # noqa: E402
from oracle import cartpole_oracle as CO  # noqa: E402
from oracle import ref_optimizer as RO  # noqa: E402

KEYS = ("residual", "barrier_param", "alpha_x", "alpha_z", "line_iters",
        "inertia_delta", "inf_pr", "inf_du", "compl", "nlp_error", "objective")


def run(m):
    r = RO.optimize(m, lambda x, a: CO.gradient(m, x, a),
                    lambda x, a: CO.hessian_values(m, x, a),
                    lambda x, a: CO.lagrangian(m, x, a),
                    lambda x: CO.objective(m, x))
    recs = []
    for it in r["records"]:
        recs.append({k: (None if it.get(k) is None or isinstance(it.get(k), str)
                         else float(it[k])) for k in KEYS})
    return dict(N=m.N, m_pole=m.m_pole, xf=m.xf, converged=r["converged"],
                iterations=r["iterations"], objective=r["objective"],
                x_norm=float(np.linalg.norm(r["x"])), records=recs)


def main(batch=6):
    cases = {"cartpole_N100_seed0": run(CartPole(N=100, seed=0))}
    B = batch_config(k=512, seed=0)
    for i in range(batch):
        cases["batch512_seed0_inst%d" % i] = run(B.inst[i])
    out = os.path.join(HERE, "ref_optimizer_cartpole.json")
    with open(out, "w") as f:
        json.dump(cases, f, indent=1)
    for k, v in cases.items():
        print(k, v["converged"], v["iterations"], v["objective"])


if __name__ == "__main__":
    main()
