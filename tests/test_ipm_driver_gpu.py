"""Whole interior-point solves of the cart-pole config (N = 100, n = 913)
with the same driver over two numeric cores: the GPU product
(DeviceBackend) and the reference's own SparseLDL + IPM vector code on the
host (oracle/host_backend.py).  Bar: both converge to KKT error <= 1e-8,
iteration counts within +-1, final objectives within 1e-8 relative."""
import numpy as np
import pytest

from amigo_b200 import ipm_driver
from amigo_b200.problems.cartpole import CartPole

pytestmark = pytest.mark.gpu


def test_cartpole_solve_device_vs_reference_core(oracle_ref):
    from oracle.host_backend import HostBackend
    m = CartPole(N=100, seed=0)
    host = ipm_driver.solve(HostBackend(m))
    prob = ipm_driver.CartPoleProblem(m, "cuda:0")
    dev = ipm_driver.solve(ipm_driver.DeviceBackend(prob, m, "cuda:0"))
    assert host["converged"] and dev["converged"]
    assert dev["kkt_error"] <= 1e-8
    assert abs(dev["iterations"] - host["iterations"]) <= 1
    assert abs(dev["objective"] - host["objective"]) <= 1e-8 * abs(host["objective"])
    # the optimum swings the pole up: theta(T) = pi
    x = dev["x"]
    assert abs(x[5 * m.N + 1] - np.pi) <= 1e-6
