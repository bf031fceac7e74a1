"""Result containers of the FDTD solvers.

Field-for-field the reference's ``EMFieldHistory`` (``src/neurosim/state.py:271-289``)
and ``EMFieldHistory3D`` (``src/neurosim/state.py:388-414``): time-major stacks of
saved frames plus the grid coordinates.  Arrays are torch tensors (fields on
the GPU, float32) unless ``simulate(..., output="numpy")`` asked for NumPy.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any


@dataclass(frozen=True)
class EMFieldHistory:
    """Time series of 2D TM field snapshots.

    Attributes:
        t: Time values, shape (n_snapshots,).
        ez: Ez snapshots, shape (n_snapshots, nx, ny).
        hx: Hx snapshots, shape (n_snapshots, nx, ny).
        hy: Hy snapshots, shape (n_snapshots, nx, ny).
        grid_x: Spatial x-coordinates.
        grid_y: Spatial y-coordinates.
    """

    t: Any
    ez: Any
    hx: Any
    hy: Any
    grid_x: Any
    grid_y: Any


@dataclass(frozen=True)
class EMFieldHistory3D:
    """Time series of 3D field snapshots.

    Attributes:
        t: Time values, shape (n_snapshots,).
        ex, ey, ez, hx, hy, hz: Snapshots, shape (n_snapshots, nx, ny, nz).
        grid_x, grid_y, grid_z: Spatial coordinates.
    """

    t: Any
    ex: Any
    ey: Any
    ez: Any
    hx: Any
    hy: Any
    hz: Any
    grid_x: Any
    grid_y: Any
    grid_z: Any


def jax_available() -> bool:
    """True when ``jax`` can be imported in this process."""
    try:
        import jax  # noqa: F401
    except Exception:
        return False
    return True


def to_jax(t):
    """A torch tensor as a JAX array.

    Through DLPack (no copy) when the JAX backend can address the tensor's
    device; otherwise through host memory (a CPU-only jaxlib cannot import a
    CUDA buffer).  The reference returns JAX arrays from ``simulate``
    (``src/neurosim/state.py:388-414``).
    """
    import jax
    import jax.numpy as jnp

    try:
        return jax.dlpack.from_dlpack(t.contiguous())
    except Exception:
        return jnp.asarray(t.detach().cpu().numpy())


def resolve_output(output: str) -> str:
    """``"auto"``: JAX arrays when JAX is importable (the reference's result
    type), torch tensors otherwise."""
    from .exceptions import ConfigurationError

    if output == "auto":
        return "jax" if jax_available() else "torch"
    if output not in ("torch", "numpy", "jax"):
        raise ConfigurationError(f"output must be 'auto', 'torch', 'numpy' or 'jax', got {output!r}")
    if output == "jax" and not jax_available():
        raise ConfigurationError("output='jax' needs the jax package")
    return output
