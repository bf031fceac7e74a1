"""Gradient-based optimisation under the reference's module path
(``src/neurosim/optimize.py``), over torch autograd and the CUDA adjoint."""

from jaxphys_b200.optimize import OptimizeResult, optimize, sensitivity  # noqa: F401
