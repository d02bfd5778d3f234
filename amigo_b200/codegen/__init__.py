"""Device code generation for component groups.

`Component` declares a component the way amigo does (inputs, data,
constants, constraints, objective, compute()); `GeneratedModel` assembles
groups of component instances into a KKT problem and compiles straight-line
CUDA evaluators of each component's Lagrangian gradient and Hessian, with
the gradient and the CSR Hessian scatter on the device.
"""
from .amigo_format import AmigoComponent, from_amigo
from .component import Component
from .expr import (acos, acosh, asin, asinh, atan, atan2, atanh, cos, cosh, exp,
                   fabs, log, log10, max2, min2, passive, sin, sinh, sqrt, tan, tanh)
from .model import GeneratedModel, Group, Slack, host_evaluator, host_evaluators, with_slacks

__all__ = ["Component", "AmigoComponent", "from_amigo", "GeneratedModel", "Group",
           "Slack", "with_slacks",
           "host_evaluator", "host_evaluators", "sin", "cos", "tan", "exp", "log", "log10", "sqrt", "tanh", "sinh", "cosh", "asin",
           "acos", "atan", "fabs", "asinh", "acosh", "atanh", "atan2", "min2", "max2",
           "passive"]
