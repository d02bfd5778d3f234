"""The benchmark models written as components for device code generation.

The cart-pole collocation problem (problems/cartpole.py) and the 2D SIMP
compliance problem (problems/simp2d.py) expressed with
amigo_b200.codegen.Component, declared the way amigo models are (inputs,
data, constraints, objective, compute(); amigo/component.py:639-706) and
assembled on the same numbering as the hand-written models, so the KKT
pattern, the gradient and the Hessian values can be compared entry by entry
with the hand-written element kernels and with the numpy restatements in
oracle/.
"""
import numpy as np

from ..codegen import Component, GeneratedModel, Group, cos, sin
from .cartpole import GRAV, L_POLE, M_CART


def _dynamics(q, u, m_pole):
    s, c = sin(q[1]), cos(q[1])
    td2 = q[3] * q[3]
    den = M_CART + m_pole * (1.0 - c * c)
    xdd = (L_POLE * m_pole * s * td2 + u + m_pole * GRAV * c * s) / den
    tdd = -(L_POLE * m_pole * c * s * td2 + u * c +
            (M_CART + m_pole) * GRAV * s) / (L_POLE * den)
    return [q[2], q[3], xdd, tdd]


class TrapezoidInterval(Component):
    """One collocation interval: node states and controls at both ends, the
    trapezoidal defects q1 - q0 - h/2 (f(q0, u0) + f(q1, u1)) = 0 and the
    trapezoidal objective h/2 (u0^2 + u1^2).  Data: the interval length and
    the pole mass (per instance, so batched instances can differ).  Outputs:
    the interval's control effort and its end state's cart position."""

    def __init__(self):
        super().__init__()
        self.add_data("h")
        self.add_data("m_pole")
        self.add_input("q0", shape=4)
        self.add_input("u0")
        self.add_input("q1", shape=4)
        self.add_input("u1")
        self.add_constraint("defect", shape=4)
        self.add_objective("effort")
        self.add_output("effort")
        self.add_output("x_end")

    def compute(self):
        h, m = self.data["h"], self.data["m_pole"]
        q0, u0 = self.inputs["q0"], self.inputs["u0"]
        q1, u1 = self.inputs["q1"], self.inputs["u1"]
        f0 = _dynamics(q0, u0, m)
        f1 = _dynamics(q1, u1, m)
        self.constraints["defect"] = [q1[j] - q0[j] - 0.5 * h * (f0[j] + f1[j])
                                      for j in range(4)]
        self.objective["effort"] = 0.5 * h * (u0 * u0 + u1 * u1)
        self.outputs["effort"] = 0.5 * h * (u0 * u0 + u1 * u1)
        self.outputs["x_end"] = q1[0]


class BoundaryState(Component):
    """A node's four states pinned by equality constraints (the targets are
    the multiplier rows' lower bounds)."""

    def __init__(self):
        super().__init__()
        self.add_input("q", shape=4)
        self.add_constraint("bc", shape=4)

    def compute(self):
        q = self.inputs["q"]
        self.constraints["bc"] = [q[j] for j in range(4)]


def cartpole_model(m):
    """GeneratedModel on the numbering of problems.cartpole.CartPole `m`."""
    data = np.stack([np.full(m.N, m.h), np.full(m.N, m.m_pole)], axis=1)
    groups = [Group(TrapezoidInterval(), m.iv, data, "interval"),
              Group(BoundaryState(), m.bv, None, "boundary")]
    return GeneratedModel(m.n, groups, m.mult, m.lower, m.upper, x0=m.x0)


# ---------------------------------------------------------------------- SIMP
class ElasticityElement(Component):
    """Plane-stress bilinear quad: equilibrium residual E(mean(rt)) K0 u of
    the element's 8 displacement DOFs, with SIMP stiffness E(r) = Emin +
    r^p (E0 - Emin) of the mean filtered nodal density.  Data: K0 (8 x 8)
    and the material constants."""

    def __init__(self, nd=8, nv=4, penalty=3.0):
        super().__init__()
        self.nd, self.nv = nd, nv
        self.add_constant("p", penalty)
        self.add_data("K0", shape=(nd, nd))
        self.add_data("E0")
        self.add_data("Emin")
        self.add_input("u", shape=nd)
        self.add_input("rt", shape=nv)
        self.add_constraint("equilibrium", shape=nd)

    def compute(self):
        K0 = self.data["K0"]
        u, rt = self.inputs["u"], self.inputs["rt"]
        E0, Emin = self.data["E0"], self.data["Emin"]
        p = self.constants["p"]
        r = sum(rt[a] for a in range(self.nv)) * (1.0 / self.nv)
        E = Emin + r ** p * (E0 - Emin)
        self.constraints["equilibrium"] = [
            E * sum(K0[i, j] * u[j] for j in range(self.nd)) for i in range(self.nd)]


class HelmholtzElement(Component):
    """Element filter residual A rt - (|e| / nv) re, A = M + r^2 K_lap."""

    def __init__(self, nv=4):
        super().__init__()
        self.nv = nv
        self.add_data("A", shape=(nv, nv))
        self.add_input("rt", shape=nv)
        self.add_input("re")
        self.add_constraint("filter", shape=nv)

    def compute(self):
        A = self.data["A"]
        rt, re = self.inputs["rt"], self.inputs["re"]
        self.constraints["filter"] = [
            sum(A[i, j] * rt[j] for j in range(self.nv)) - re * (1.0 / self.nv)
            for i in range(self.nv)]


class VolumeTerm(Component):
    """One element's share re / nelems of the volume constraint (its
    multiplier is one variable shared by every element)."""

    def __init__(self):
        super().__init__()
        self.add_data("coef")
        self.add_input("re")
        self.add_constraint("volume")

    def compute(self):
        self.constraints["volume"] = self.inputs["re"] * self.data["coef"]


class VolumeBound(Component):
    """The constant and slack part of the volume constraint:
    -volfrac - s (added to the same multiplier row as the VolumeTerms)."""

    def __init__(self, volfrac):
        super().__init__()
        self.add_constant("volfrac", volfrac)
        self.add_input("s")
        self.add_constraint("volume")

    def compute(self):
        self.constraints["volume"] = -self.constants["volfrac"] - self.inputs["s"]


class PointLoad(Component):
    """Compliance F u of the loaded DOF and the load's share -F of its
    equilibrium residual."""

    def __init__(self):
        super().__init__()
        self.add_data("F")
        self.add_input("u")
        self.add_constraint("load")
        self.add_objective("compliance")

    def compute(self):
        F = self.data["F"]
        self.constraints["load"] = -F
        self.objective["compliance"] = F * self.inputs["u"]


def simp2d_model(m):
    """GeneratedModel on the numbering of problems.simp2d.Simp2D `m`."""
    from .simp2d import E0, EMIN, PENALTY
    ne = m.nelems
    nd, nv = m.K0.shape[0], m.A.shape[0]
    edata = np.concatenate([np.broadcast_to(m.K0.ravel(), (ne, nd * nd)),
                            np.full((ne, 1), E0), np.full((ne, 1), EMIN)], axis=1)
    # elasticity: [u (nd), rt (nv) | lam (nd)] = m.ev
    fdata = np.broadcast_to(m.A.ravel(), (ne, nv * nv))
    # filter: [rt (nv), re | mu (nv)] = m.fv
    re = m.re0 + np.arange(ne)
    vidx = np.stack([re, np.full(ne, m.nu0)], axis=1)
    load = np.nonzero(m.f)[0]
    lidx = np.stack([load, m.lam0 + (load - m.u0)], axis=1)
    groups = [Group(ElasticityElement(nd, nv, PENALTY), m.ev, edata, "elasticity"),
              Group(HelmholtzElement(nv), m.fv, fdata, "filter"),
              Group(VolumeTerm(), vidx, np.full((ne, 1), 1.0 / ne), "volume"),
              Group(VolumeBound(m.volfrac), np.array([[m.s0, m.nu0]]), None, "volume_bound"),
              Group(PointLoad(), lidx, m.f[load][:, None], "load")]
    return GeneratedModel(m.n, groups, m.mult, m.lower, m.upper, fixed=m.fixed,
                          x0=m.initial_point())
