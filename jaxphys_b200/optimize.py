"""Gradient-based optimisation driver over the engine's adjoint.

The reference's ``optimize`` (``src/neurosim/optimize.py:49-207``) minimises
a scalar objective with gradient descent or Adam, taking gradients with
``jax.grad``.  Here the same loop runs over torch autograd, so an objective
built on :func:`jaxphys_b200.em.adjoint.probe_traces` differentiates through
the hand-written CUDA adjoint of the FDTD step (sqrt(T) checkpointing):

    >>> theta0 = torch.randn(32, 32, 32, device="cuda")
    >>> def objective(theta):                 # inverse design, config 4 style
    ...     eps = torch.ones(grid.size, device="cuda")
    ...     eps[region] = 1 + 11 * torch.sigmoid(theta)
    ...     return -(probe_traces(grid, eps, 2000) ** 2).sum()
    >>> res = optimize(objective, theta0, learning_rate=0.05, max_iterations=20,
    ...                method="adam")

``sensitivity`` is the reference's Jacobian helper (``optimize.py:210-228``).

Same arguments, defaults, update rules and stopping test as the reference:
gradient descent x <- x - lr g; Adam with beta1 = 0.9, beta2 = 0.999,
eps = 1e-8 and bias correction (``optimize.py:142-207``); convergence when
the gradient's 2-norm drops below ``tolerance`` (checked before the update,
``optimize.py:108-119,180-189``).
"""

from __future__ import annotations

import logging
from dataclasses import dataclass
from typing import Any

import torch

logger = logging.getLogger(__name__)


@dataclass(frozen=True)
class OptimizeResult:
    """Result of an optimization run (``optimize.py:30-46``).

    Attributes:
        x: Optimal parameter value.
        fun: Objective function value at optimum.
        n_iterations: Number of iterations performed.
        converged: Whether the optimizer converged.
        trajectory: History of parameter values (if tracked).
    """

    x: torch.Tensor
    fun: float
    n_iterations: int
    converged: bool
    trajectory: torch.Tensor | None = None


def _grad(objective, x: torch.Tensor) -> torch.Tensor:
    xr = x.detach().requires_grad_(True)
    val = objective(xr)
    (g,) = torch.autograd.grad(val, xr)
    return g.detach()


def _value(objective, x: torch.Tensor) -> float:
    with torch.no_grad():
        return float(objective(x.detach()))


def optimize(
    objective: Any,
    initial_guess,
    learning_rate: float = 0.01,
    max_iterations: int = 1000,
    tolerance: float = 1e-8,
    method: str = "gradient_descent",
    track_trajectory: bool = False,
) -> OptimizeResult:
    """Minimize a scalar torch-differentiable objective (``optimize.py:49-139``).

    Args:
        objective: Scalar-valued function of a tensor, differentiable by torch
            autograd (e.g. through ``probe_traces``).
        initial_guess: Starting parameter value (tensor or float).
        learning_rate: Step size for optimization.
        max_iterations: Maximum number of iterations.
        tolerance: Convergence threshold on gradient norm.
        method: "gradient_descent" or "adam".
        track_trajectory: Whether to save parameter history.
    """
    if method not in ("gradient_descent", "adam"):
        raise ValueError(f"unknown method {method!r}")
    # Python numbers, lists and arrays become float64 as in the reference
    # (optimize.py:83, jnp.asarray(..., float64)); a floating tensor keeps its
    # dtype and device (e.g. float32 parameters of a CUDA objective)
    if isinstance(initial_guess, torch.Tensor) and torch.is_floating_point(initial_guess):
        x = initial_guess.detach().clone()
    else:
        x = torch.as_tensor(initial_guess, dtype=torch.float64).detach().clone()
    logger.info("Starting optimization: method=%s, lr=%.2e, max_iter=%d", method,
                learning_rate, max_iterations)
    traj = [x.clone()] if track_trajectory else []

    def result(n, converged):
        return OptimizeResult(x=x, fun=_value(objective, x), n_iterations=n, converged=converged,
                              trajectory=torch.stack(traj) if track_trajectory else None)

    if method == "adam":
        beta1, beta2, eps = 0.9, 0.999, 1e-8
        m = torch.zeros_like(x)
        v = torch.zeros_like(x)
        for i in range(1, max_iterations + 1):
            g = _grad(objective, x)
            if float(torch.sqrt(torch.sum(g * g))) < tolerance:
                return result(i, True)
            m = beta1 * m + (1 - beta1) * g
            v = beta2 * v + (1 - beta2) * g * g
            m_hat = m / (1 - beta1 ** i)
            v_hat = v / (1 - beta2 ** i)
            x = x - learning_rate * m_hat / (torch.sqrt(v_hat) + eps)
            if track_trajectory:
                traj.append(x.clone())
        return result(max_iterations, False)

    for i in range(max_iterations):
        g = _grad(objective, x)
        grad_norm = float(torch.sqrt(torch.sum(g * g)))
        if grad_norm < tolerance:
            logger.info("Converged at iteration %d, grad_norm=%.2e", i, grad_norm)
            return result(i, True)
        x = x - learning_rate * g
        if track_trajectory:
            traj.append(x.clone())
    logger.warning("Optimization did not converge after %d iterations", max_iterations)
    return result(max_iterations, False)


def sensitivity(simulation_fn: Any, params) -> torch.Tensor:
    """Jacobian d(outputs)/d(params) of a simulation (``optimize.py:210-228``).

    ``params`` becomes a float64 tensor (as the reference's ``jnp.asarray(...,
    dtype=float64)``); the Jacobian comes from torch autograd, so a
    ``simulation_fn`` built on ``probe_traces`` differentiates through the
    CUDA adjoint.  Shape: outputs' shape + params' shape.
    """
    p = torch.as_tensor(params, dtype=torch.float64).detach()
    return torch.autograd.functional.jacobian(simulation_fn, p)
