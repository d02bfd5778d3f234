"""Device code generation for component groups, GPU part: the generated
gradient and Hessian kernels against the hand-written element kernels of
the same models (cartpole.cu, fem_simp.cu) on the same CSR pattern, within
FP64 rounding (different operation order: rtol 1e-13 of the largest
entry), deterministic (bit-identical on a second evaluation), and a whole
interior-point solve of the cart-pole problem through the generated model
reaching the hand-written model's iterations and objective."""
import numpy as np
import pytest
import torch

from amigo_b200.problems import components as C
from amigo_b200.problems.cartpole import CartPole
from amigo_b200.problems.simp2d import Simp2D

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _compare(m, gen, hand, x, alpha):
    xd = torch.from_numpy(x).to(DEV)
    g1 = torch.zeros(m.n, dtype=torch.float64, device=DEV)
    g2 = torch.zeros_like(g1)
    gen.gradient(xd, alpha, g1)
    hand.gradient(xd, alpha, g2)
    a, b = g1.cpu().numpy(), g2.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-13 * max(1.0, np.abs(b).max())
    v1 = torch.full((m.nnz,), 3.0, dtype=torch.float64, device=DEV)
    v2 = torch.zeros_like(v1)
    gen.hessian(xd, alpha, v1)
    hand.hessian(xd, alpha, v2)
    a, b = v1.cpu().numpy(), v2.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-13 * max(1.0, np.abs(b).max())
    v3 = torch.zeros_like(v1)
    gen.hessian(xd, alpha, v3)
    assert torch.equal(v1, v3)


def test_cartpole_generated_kernels_match_hand_written():
    m = CartPole(N=100, seed=0)
    G = C.cartpole_model(m)
    x = m.x0 + 0.05 * np.random.RandomState(2).randn(m.n)
    _compare(m, G.device_model(DEV), m.device_model(DEV), x, 0.8)


def test_simp2d_generated_kernels_match_hand_written():
    m = Simp2D(40, 20, seed=1)
    G = C.simp2d_model(m)
    r = np.random.RandomState(3)
    x = r.randn(m.n) * 0.3
    x[m.rt0:m.rt0 + m.nnodes] = 0.2 + 0.6 * r.rand(m.nnodes)
    x[m.re0:m.re0 + m.nelems] = 0.2 + 0.6 * r.rand(m.nelems)
    _compare(m, G.device_model(DEV), m.device_model(DEV), x, 1.0)


def test_cartpole_ipm_through_generated_model():
    from amigo_b200 import ipm_driver
    m = CartPole(N=100, seed=0)
    G = C.cartpole_model(m)
    hand = ipm_driver.solve(ipm_driver.DeviceBackend(
        ipm_driver.CartPoleProblem(m, DEV), m, DEV))
    gen = ipm_driver.solve(ipm_driver.DeviceBackend(
        ipm_driver.GeneratedProblem(G, DEV), G, DEV))
    assert gen["converged"] and hand["converged"]
    assert abs(gen["iterations"] - hand["iterations"]) <= 1
    assert abs(gen["objective"] - hand["objective"]) <= 1e-8 * abs(hand["objective"])
