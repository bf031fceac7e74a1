"""Differentiable probe readout of the 3D solver (extension).

``probe_traces(grid, eps_r, n_steps)`` runs the grid from rest with the
per-cell relative permittivity ``eps_r`` (a CUDA float32 tensor of the grid
shape) and returns the probe traces (n_steps, n_probes).  It is a
``torch.autograd.Function``: ``backward`` runs the hand-written discrete
adjoint (time-reversed Yee step, sqrt(T) checkpointing) in
``jaxphys_b200/csrc/fdtd3d_adjoint.cuh`` and returns dJ/d(eps_r), so any torch
objective of the traces (and any torch parametrisation of eps_r, e.g.
``1 + 11*sigmoid(theta)`` on a design region) differentiates end to end.

The reference differentiates only through ``jax.grad`` on its generic
optimiser (``src/neurosim/optimize.py:84``); through ``EMGrid3D.simulate`` that
would store every step of the ``lax.scan``.  A ``jax.custom_vjp`` wrapper with
the same forward/backward pair is provided when JAX is importable.
"""

from __future__ import annotations

import torch


class _ProbeTraces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eps_r, grid, n_steps, checkpoint_every):
        grid.set_permittivity_device(eps_r.detach())
        traces = grid.adjoint_forward(n_steps, checkpoint_every)
        ctx.grid = grid
        return traces

    @staticmethod
    def backward(ctx, grad_traces):
        grad_eps = ctx.grid.adjoint_backward(grad_traces)
        return grad_eps, None, None, None


def probe_traces(grid, eps_r: torch.Tensor, n_steps: int, checkpoint_every: int | None = None):
    """Probe traces of ``grid`` run from rest for ``n_steps`` with ``eps_r``;
    differentiable with respect to ``eps_r`` (see module docstring)."""
    if not eps_r.is_cuda:
        raise ValueError("eps_r must be a CUDA tensor")
    return _ProbeTraces.apply(eps_r, grid, int(n_steps), checkpoint_every)


def jax_probe_traces(grid, n_steps: int, checkpoint_every: int | None = None):
    """``jax.custom_vjp`` version (only when JAX is installed): returns a
    function eps_r -> traces whose VJP is the same adjoint."""
    import jax  # noqa: F401  (raises ImportError when JAX is absent)
    import jax.dlpack

    @jax.custom_vjp
    def f(eps_r):
        return _fwd(eps_r)[0]

    def _fwd(eps_r):
        t = torch.from_dlpack(eps_r)
        grid.set_permittivity_device(t)
        tr = grid.adjoint_forward(n_steps, checkpoint_every)
        return jax.dlpack.from_dlpack(tr), None

    def _bwd(_, g):
        ge = grid.adjoint_backward(torch.from_dlpack(g))
        return (jax.dlpack.from_dlpack(ge),)

    f.defvjp(_fwd, _bwd)
    return f
